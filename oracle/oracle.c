/* oracle.c : CPU restatement of the Opticks simulate path, used ONLY as test infrastructure
 * (the checker in tests/, the smoke check and the CPU baseline leg of bench.py).  It is never
 * part of the product path.
 *
 * What it restates (paths within simoncblyth/opticks):
 *   CSG intersection            see oracle_csg.inc (CSG/csg_intersect_*.h)
 *   closest hit over instances  CSGOptiX/CSGOptiX7.cu:776-967 (IS/CH semantics), brute force
 *   bounce loop + seq           CSGOptiX/CSGOptiX7.cu:432-530, sysrap/sctx.h:134-185, sysrap/sseq.h:174-184
 *   propagate physics           qudarap/qsim.h:180-201, 433-866, 1001-1208, 1680-1758, 1988-2093, 2229-2338
 *   fill_state                  qudarap/qbnd.h:108-224
 *   generation                  sysrap/storch.h:192-520, qudarap/qscint.h:66-258, qudarap/qcerenkov.h:56-320
 *   hit selection               sysrap/sphoton.h:1272-1278 (all bits of the hit mask)
 * Texture lookups emulate CUDA hardware linear filtering (normalized coordinates, wrap address
 * mode, weights with 8 fractional bits, as the CUDA programming guide describes texture
 * fetching).  Random numbers are consumed from precooked per-photon uniform streams dumped by
 * the GPU (the reference does the same with sysrap/s_seq.h), so the oracle needs no cuRAND.
 * Arithmetic is IEEE FP32 with libm; the CUDA engine uses fast-math intrinsics, so comparisons
 * allow ulp-level differences and tally rare decision flips.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_F 3.14159265358979323846f

typedef struct {
    const float* node;
    const float* itra;
    int polish;
    const float* plan;          /* (Nl,4) convex polyhedron planes, or NULL */
} oracle_csg;

/* Kensler single-hit CSG actions: 0 miss, 1 return A, 2 return B, 3 return flipped B,
 * 4 loop A, 5 loop B.  Table [op-1][aCloser][3*stateA+stateB], states Enter 0, Exit 1, Miss 2 */
static const unsigned char ACTION[3][2][9] = {
    /* union        B closer                        A closer */
    { { 2, 2, 1, 5, 1, 1, 2, 2, 0 }, { 1, 4, 1, 1, 2, 1, 2, 2, 0 } },
    /* intersection */
    { { 5, 5, 0, 2, 2, 0, 0, 0, 0 }, { 4, 1, 0, 4, 1, 0, 0, 0, 0 } },
    /* difference   */
    { { 5, 5, 1, 3, 3, 1, 0, 0, 0 }, { 1, 4, 1, 1, 4, 1, 0, 0, 0 } },
};

int oracle_csg_action(int op, int sa, int sb, int a_closer)
{
    if (op < 1 || op > 3) return 0;
    return ACTION[op - 1][a_closer ? 1 : 0][3 * sa + sb];
}

static double q4(const double* c, double u) { return (((u + c[3]) * u + c[2]) * u + c[1]) * u + c[0]; }
static double q4d(const double* c, double u) { return ((4 * u + 3 * c[3]) * u + 2 * c[2]) * u + c[1]; }

/* smallest real root of the monic quartic in (lo,hi] */
static int oracle_quartic_first_root(const double* c, double lo, double hi, double* root)
{
    /* stationary points : 4u^3 + 3c3 u^2 + 2c2 u + c1 = 0 */
    double a = 0.75 * c[3], b = 0.5 * c[2], cc = 0.25 * c[1];
    double a3 = a / 3, p = b - a * a3, q = 2 * a3 * a3 * a3 - a3 * b + cc;
    double disc = 0.25 * q * q + p * p * p / 27;
    double crit[3];
    int nc;
    if (disc > 0) { double s = sqrt(disc); crit[0] = cbrt(-0.5 * q + s) + cbrt(-0.5 * q - s) - a3; nc = 1; }
    else if (p == 0) { crit[0] = -a3; nc = 1; }
    else {
        double m = 2 * sqrt(-p / 3), arg = 3 * q / (p * m);
        arg = arg > 1 ? 1 : (arg < -1 ? -1 : arg);
        double th = acos(arg) / 3, tp = 2.0943951023931954923;
        crit[0] = m * cos(th) - a3; crit[1] = m * cos(th - tp) - a3; crit[2] = m * cos(th - 2 * tp) - a3;
        nc = 3;
        for (int i = 0; i < 3; i++) for (int j = i + 1; j < 3; j++) if (crit[j] < crit[i]) { double t = crit[i]; crit[i] = crit[j]; crit[j] = t; }
    }
    double e[5];
    int ne = 0;
    e[ne++] = lo;
    for (int i = 0; i < nc; i++) if (crit[i] > lo && crit[i] < hi) e[ne++] = crit[i];
    e[ne++] = hi;
    for (int i = 0; i + 1 < ne; i++) {
        double x0 = e[i], x1 = e[i + 1], f0 = q4(c, x0), f1 = q4(c, x1);
        if (f0 == 0 && i > 0) { *root = x0; return 1; }
        if ((f0 < 0) == (f1 < 0) && f1 != 0) continue;
        /* plain bisection to full double precision (independent of the engine's Newton) */
        for (int it = 0; it < 200 && x1 - x0 > 1e-13 * (1 + fabs(x0)); it++) {
            double xm = 0.5 * (x0 + x1), fm = q4(c, xm);
            if (fm == 0) { x0 = x1 = xm; break; }
            if ((fm < 0) == (f0 < 0)) { x0 = xm; f0 = fm; } else { x1 = xm; }
        }
        (void)q4d;
        *root = 0.5 * (x0 + x1);
        return 1;
    }
    return 0;
}

#define REAL float
#define SFX _f
#include "oracle_csg.inc"
#undef REAL
#undef SFX
#define REAL double
#define SFX _d
#include "oracle_csg.inc"
#undef REAL
#undef SFX

/* ------------------------------------------------------------------ CSG scan entry points */
/* rays SoA (6,n); out (n,4) normal.xyz,t (t=0 miss); returns OR of evaluator errors */
int oracle_csg_scan(const float* node, const float* itra, const float* plan, int root, float tmin, const float* rays,
                    long long n, float* out, int use_double, int polish)
{
    oracle_csg g = { node, itra, polish, plan };
    int err_all = 0;
#pragma omp parallel for schedule(static) reduction(| : err_all)
    for (long long i = 0; i < n; i++) {
        int err = 0;
        if (use_double) {
            vec_d o = mk_d(rays[i], rays[n + i], rays[2 * n + i]);
            vec_d d = mk_d(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
            double is[4];
            int v = prim_d(is, &g, root, tmin, o, d, &err);
            for (int k = 0; k < 4; k++) out[4 * i + k] = v ? (float)is[k] : 0.f;
        } else {
            vec_f o = mk_f(rays[i], rays[n + i], rays[2 * n + i]);
            vec_f d = mk_f(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
            float is[4];
            int v = prim_f(is, &g, root, tmin, o, d, &err);
            for (int k = 0; k < 4; k++) out[4 * i + k] = v ? is[k] : 0.f;
        }
        err_all |= err;
    }
    return err_all;
}

/* FP64 distance along each ray (t, 0 for miss) for intersection-distance error statistics */
int oracle_csg_scan_t64(const float* node, const float* itra, const float* plan, int root, float tmin, const float* rays,
                        long long n, double* t)
{
    oracle_csg g = { node, itra, 0, plan };
    int err_all = 0;
#pragma omp parallel for schedule(static) reduction(| : err_all)
    for (long long i = 0; i < n; i++) {
        int err = 0;
        vec_d o = mk_d(rays[i], rays[n + i], rays[2 * n + i]);
        vec_d d = mk_d(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
        double is[4];
        int v = prim_d(is, &g, root, tmin, o, d, &err);
        t[i] = v ? is[3] : 0.0;
        err_all |= err;
    }
    return err_all;
}

/* the same with FP64 rays (SoA (6,n) doubles): rays carried into a prim's frame in double keep
   the world ray exactly, so the distance error measured against it is the FP32 path's alone */
int oracle_csg_scan_t64d(const float* node, const float* itra, const float* plan, int root, double tmin, const double* rays,
                         long long n, double* t)
{
    oracle_csg g = { node, itra, 0, plan };
    int err_all = 0;
#pragma omp parallel for schedule(static) reduction(| : err_all)
    for (long long i = 0; i < n; i++) {
        int err = 0;
        vec_d o = mk_d(rays[i], rays[n + i], rays[2 * n + i]);
        vec_d d = mk_d(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
        double is[4];
        int v = prim_d(is, &g, root, tmin, o, d, &err);
        t[i] = v ? is[3] : 0.0;
        err_all |= err;
    }
    return err_all;
}

/* ------------------------------------------------------------------ textures */
typedef struct { float x, y, z, w; } f4;

/* hardware-style linear filtering: texel coordinate x*W-0.5, 8 fractional weight bits, wrap */
static void tex_setup(float c, int W, int* i0, int* i1, float* a)
{
    float xb = c * (float)W - 0.5f;
    float fl = floorf(xb);
    float fr = xb - fl;
    *a = (float)((int)(fr * 256.0f + 0.5f)) / 256.0f;
    int i = (int)fl;
    *i0 = ((i % W) + W) % W;
    *i1 = (((i + 1) % W) + W) % W;
}

static f4 tex2d_f4(const float* data, int W, int H, float x, float y)
{
    int x0, x1, y0, y1;
    float ax, ay;
    tex_setup(x, W, &x0, &x1, &ax);
    tex_setup(y, H, &y0, &y1, &ay);
    const float* t00 = data + 4 * ((size_t)y0 * W + x0);
    const float* t10 = data + 4 * ((size_t)y0 * W + x1);
    const float* t01 = data + 4 * ((size_t)y1 * W + x0);
    const float* t11 = data + 4 * ((size_t)y1 * W + x1);
    float r[4];
    for (int k = 0; k < 4; k++)
        r[k] = (1 - ax) * (1 - ay) * t00[k] + ax * (1 - ay) * t10[k] + (1 - ax) * ay * t01[k] + ax * ay * t11[k];
    f4 o = { r[0], r[1], r[2], r[3] };
    return o;
}

static float tex2d_f1(const float* data, int W, int H, float x, float y)
{
    int x0, x1, y0, y1;
    float ax, ay;
    tex_setup(x, W, &x0, &x1, &ax);
    tex_setup(y, H, &y0, &y1, &ay);
    return (1 - ax) * (1 - ay) * data[(size_t)y0 * W + x0] + ax * (1 - ay) * data[(size_t)y0 * W + x1]
         + (1 - ax) * ay * data[(size_t)y1 * W + x0] + ax * ay * data[(size_t)y1 * W + x1];
}

/* QPlanck's table (qudarap/QPlanck.cc:36-48): Planck's law at 4096 wavelengths over 80-800 nm at
   6500 K (sysrap/sblackbody.h:77-116), trapezoid integral / last (NP::trapz, NP::divide_by_last),
   inverted at y = j/4096 by the first bin with y0 <= y < y1 and linear interpolation
   (NP::MakeICDF hd_factor 0, NP::pdomain), in double, narrowed to float. */
int oracle_planck_icdf(float* out, int n)
{
    enum { NI = 4096, NU = 4096 };
    if (!out || n < NU) return -1;
    static double x[NI], y[NI], cdf[NI];
    const double T = 6500.0, nm0 = 80.0, nm1 = 800.0;
    const double h = 6.62606957e-34, c = 299792458.0, k = 1.3806488e-23;
    const double a = 2.0 * h * c * c, b = h * c / k;
    for (int i = 0; i < NI; i++) {
        x[i] = nm0 + (nm1 - nm0) * (double)i / (double)(NI - 1);
        double wlm = x[i] * 1e-9;
        y[i] = (a * pow(wlm, -5.0)) / (exp(b / (wlm * T)) - 1.0);
    }
    cdf[0] = 0.0;
    for (int i = 0; i < NI - 1; i++) cdf[i + 1] = cdf[i] + (x[i + 1] - x[i]) * (y[i] + y[i + 1]) * 0.5;
    double last = cdf[NI - 1];
    if (last != 0.0) for (int i = 0; i < NI; i++) cdf[i] /= last;
    for (int j = 0; j < NU; j++) {
        double yv = (double)j / (double)NU, xv = x[0];
        if (yv <= cdf[0]) xv = x[0];
        else if (yv >= cdf[NI - 1]) xv = x[NI - 1];
        else
            for (int i = 0; i < NI - 1; i++) {
                double y0 = cdf[i], y1 = cdf[i + 1], dy = y1 - y0;
                if (y0 <= yv && yv < y1) { xv = x[i]; if (dy > 0.0) xv += (yv - y0) * (x[i + 1] - x[i]) / dy; break; }
            }
        out[j] = (float)xv;
    }
    return 0;
}

/* ------------------------------------------------------------------ scene */
typedef struct {
    const float* node;          /* (Nn,4,4) */
    const float* itra;          /* (Nt,4,4) */
    const float* inst_inv;      /* (Ni,4,4) world->object rows */
    const int* pair_inst;       /* (Np) instance of each (instance,prim) pair */
    const int* pair_node;       /* (Np) root node of the prim */
    const unsigned* pair_gpbd;  /* (Np) globalPrimIdx<<16|boundary */
    const unsigned* pair_iiid;  /* (Np) iindex<<16|identity */
    int num_pair;
    const float* bnd;           /* (H=nb*8, W=num_wl, 4) */
    int bnd_w, bnd_h;
    float nm0, nms;
    const unsigned* optical;    /* (nb*4,4) */
    const float* icdf;          /* (3, width) */
    int icdf_w, icdf_h, hd_factor;
    int max_bounce;
    float max_time, tmin, tmin0;
    unsigned eps0_mask, hit_mask;
    int polish;
    const float* pair_bbox;     /* (Np,6) padded world boxes, or NULL for no culling */
    const float* plan;          /* (Nl,4) convex polyhedron planes, or NULL */
    const float* input_photon;  /* (num_input,4,4) sphoton rows for INPUT_PHOTON gensteps, or NULL */
    long long num_input;
    const float* planck;        /* (4096) black-body wavelength ICDF, or NULL */
} oracle_scene;

typedef struct { const float* u; int n; int k; int over; } ustream;
static float U(ustream* s)
{
    if (s->k >= s->n) { s->over = 1; return 0.5f; }
    return s->u[s->k++];
}

typedef struct { float x, y, z; } v3;
static inline v3 V(float x, float y, float z) { v3 r = { x, y, z }; return r; }
static inline v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(float s, v3 a) { return V(s * a.x, s * a.y, s * a.z); }
static inline float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float len3(v3 a) { return sqrtf(dot3(a, a)); }
static inline v3 norm3(v3 a) { float il = 1.0f / sqrtf(dot3(a, a)); return mul(il, a); }

static void rotate_uz(v3* d, v3 u)
{
    float up = u.x * u.x + u.y * u.y;
    if (up > 0.f) {
        up = sqrtf(up);
        float px = d->x, py = d->y, pz = d->z;
        d->x = (u.x * u.z * px - u.y * py) / up + u.x * pz;
        d->y = (u.y * u.z * px + u.x * py) / up + u.y * pz;
        d->z = -up * px + u.z * pz;
    } else if (u.z < 0.f) { d->x = -d->x; d->z = -d->z; }
}

typedef struct {
    v3 pos; float time;
    v3 mom; unsigned hitcount_iindex;
    v3 pol; float wavelength;
    unsigned obf, identity, index, flagmask;
} photon_t;

static void set_flag(photon_t* p, unsigned f) { p->obf = (p->obf & 0xffff0000u) | (f & 0xffffu); p->flagmask |= f; }
static void zero_flags(photon_t* p) { p->obf = 0; p->identity = 0; p->index = 0; p->flagmask = 0; p->hitcount_iindex = 0; }

static f4 bnd_lookup(const oracle_scene* S, float nm, unsigned line, unsigned k)
{
    float fx = (nm - S->nm0) / S->nms;
    float x = (fx + 0.5f) / (float)S->bnd_w;
    unsigned iy = 2 * line + k;
    float y = ((float)iy + 0.5f) / (float)S->bnd_h;
    return tex2d_f4(S->bnd, S->bnd_w, S->bnd_h, x, y);
}

static float scint_wl(const oracle_scene* S, float u0)
{
    if (!S->icdf) return 0.f;
    float x, y;
    if (S->hd_factor == 20) {
        int l = u0 < 0.05f, r = u0 > 0.95f;
        x = l ? u0 * 20.f : (r ? (u0 - 0.95f) * 20.f : u0);
        y = l ? 1.5f / 3.f : (r ? 2.5f / 3.f : 0.5f / 3.f);
    } else if (S->hd_factor == 10) {
        int l = u0 < 0.1f, r = u0 > 0.9f;
        x = l ? u0 * 10.f : (r ? (u0 - 0.9f) * 10.f : u0);
        y = l ? 1.5f / 3.f : (r ? 2.5f / 3.f : 0.5f / 3.f);
    } else { x = u0; y = 0.5f / 3.f; }
    return tex2d_f1(S->icdf, S->icdf_w, S->icdf_h, x, y);
}

static v3 uniform_sphere(float u0, float u1)
{
    float phi = u0 * 2.f * PI_F, ct = 2.f * u1 - 1.f, st = sqrtf(1.f - ct * ct);
    return V(cosf(phi) * st, sinf(phi) * st, ct);
}

/* ------------------------------------------------------------------ generation */
static void gen_torch(photon_t* p, ustream* r, const float* g, unsigned long long pid)
{
    unsigned type, nph;
    memcpy(&type, g + 23, 4);
    memcpy(&nph, g + 3, 4);
    v3 gpos = V(g[4], g[5], g[6]), gmom = V(g[8], g[9], g[10]);
    float zx = g[16], zy = g[17], ax = g[18], ay = g[19], radius = g[20], dist = g[21];
    p->wavelength = g[15];
    p->time = g[7];
    if (type == 1) { /* disc */
        p->mom = gmom;
        float uz = zx + U(r) * (zy - zx), ua = ax + U(r) * (ay - ax);
        float rr = radius * uz, phi = 2.f * PI_F * ua, s = sinf(phi), c = cosf(phi);
        p->pos = V(rr * c, rr * s, 0.f); rotate_uz(&p->pos, p->mom); p->pos = add(p->pos, gpos);
        p->pol = V(s, -c, 0.f); rotate_uz(&p->pol, p->mom);
    } else if (type == 7 || type == 64) { /* sphere, sphere with random polarisation */
        float uz = zx + U(r) * (zy - zx), ua = ax + U(r) * (ay - ax);
        float phi = 2.f * PI_F * ua, s = sinf(phi), c = cosf(phi);
        float ct = 1.f - 2.0f * uz, st = sqrtf(1.0f - ct * ct), flip = copysignf(1.f, radius), rad = fabsf(radius);
        p->mom = V(flip * st * c, flip * st * s, flip * ct);
        p->pos = V(st * c * rad, st * s * rad, ct * rad);
        float ft = type == 64 ? U(r) : dist;
        float ph = 2.f * PI_F * ft;
        p->pol = V(cosf(ph), sinf(ph), 0.f); rotate_uz(&p->pol, p->mom);
    } else if (type == 3) { /* point */
        p->mom = gmom;
        p->pos = gpos;
        p->pol = V(0.f, -1.f, 0.f); rotate_uz(&p->pol, p->mom);
    } else if (type == 2) { /* line */
        p->mom = gmom;
        float frac = (float)pid / (float)nph, sf = 2.f * (frac - 0.5f), rr = radius * sf;
        p->pos = V(rr, 0.f, 0.f); rotate_uz(&p->pos, p->mom); p->pos = add(p->pos, gpos);
        p->pol = V(0.f, -1.f, 0.f); rotate_uz(&p->pol, p->mom);
    }
    zero_flags(p);
    set_flag(p, 0x4);
}

/* scarrier::generate sysrap/scarrier.h: genstep rows 2-5, moved 10 mm in y per photon index */
static void gen_carrier(photon_t* p, const float* g, unsigned long long pid)
{
    p->pos.x = g[8]; p->pos.y = g[9] + (float)pid * 10.f; p->pos.z = g[10]; p->time = g[11];
    p->mom.x = g[12]; p->mom.y = g[13]; p->mom.z = g[14]; memcpy(&p->hitcount_iindex, g + 15, 4);
    p->pol.x = g[16]; p->pol.y = g[17]; p->pol.z = g[18]; p->wavelength = g[19];
    memcpy(&p->obf, g + 20, 4); memcpy(&p->identity, g + 21, 4); memcpy(&p->index, g + 22, 4); memcpy(&p->flagmask, g + 23, 4);
    set_flag(p, 0x4);
}

static void gen_scint(photon_t* p, ustream* r, const float* g, const oracle_scene* S)
{
    float u0 = U(r), u1 = U(r), u2 = U(r), u3 = U(r);
    float ct = 1.f - 2.f * u0, st = sqrtf((1.f - ct) * (1.f + ct));
    float phi = 2.f * PI_F * u1, sp = sinf(phi), cp = cosf(phi);
    p->mom = V(st * cp, st * sp, ct);
    p->pol = V(ct * cp, ct * sp, -st);
    phi = 2.f * PI_F * u2; sp = sinf(phi); cp = cosf(phi);
    p->pol = norm3(add(mul(cp, p->pol), mul(sp, cross3(p->mom, p->pol))));
    p->wavelength = scint_wl(S, u3);
    float charge = g[13];
    float frac = charge == 0.f ? 1.f : U(r);
    p->pos = add(V(g[4], g[5], g[6]), mul(frac, V(g[8], g[9], g[10])));
    float u4 = U(r);
    p->time = g[7] + (frac * g[11] / g[15] - g[20] * logf(u4));
    zero_flags(p);
    set_flag(p, 0x2);
}

static void gen_cerenkov(photon_t* p, ustream* r, const float* g, const oracle_scene* S)
{
    unsigned matline;
    memcpy(&matline, g + 2, 4);
    v3 dp = V(g[8], g[9], g[10]);
    v3 p0 = norm3(dp);
    float bi = g[16], wmin = g[17], wmax = g[18], max_sin2 = g[20], m1 = g[21], m2 = g[22], post = g[23], pre = g[15];
    float wl = 0, ct = 0, s2 = 0, u1 = 0;
    int count = 0;
    do {
        float u0 = U(r);
        float w = wmin + u0 * (wmax - wmin);
        wl = wmin * wmax / w;
        f4 pr = bnd_lookup(S, wl, matline, 0);
        ct = bi / pr.x;
        s2 = fmaxf(0.f, (1.f - ct) * (1.f + ct));
        u1 = U(r);
        count++;
    } while (u1 * max_sin2 > s2 && count < 100 && !r->over);
    float st = sqrtf(s2), u0 = U(r), phi = 2.f * PI_F * u0, sp = sinf(phi), cp = cosf(phi);
    p->mom = V(st * cp, st * sp, ct); rotate_uz(&p->mom, p0);
    p->pol = V(ct * cp, ct * sp, -st); rotate_uz(&p->pol, p0);
    p->wavelength = wl;
    float frac, delta, N, NP, mx = fmaxf(m1, m2), dn = m1 - m2;
    do { frac = U(r); delta = frac * g[11]; NP = m1 - frac * dn; N = U(r) * mx; } while (N > NP && !r->over);
    float mid = pre + frac * (post - pre) * 0.5f;
    p->time = g[7] + delta / mid;
    p->pos = add(V(g[4], g[5], g[6]), mul(frac, dp));
    zero_flags(p);
    set_flag(p, 0x1);
}

/* ------------------------------------------------------------------ closest hit */
typedef struct { v3 n; float t; float lposcost; unsigned gpbd, iiid; } prd_t;

static int trace(const oracle_scene* S, v3 o, v3 d, float tmin, prd_t* prd, int* err)
{
    float best = 1000000.f;
    int bi = -1;
    float bis[4] = { 0, 0, 0, 0 };
    float blc = 0.f;
    oracle_csg g = { S->node, S->itra, S->polish, S->plan };
    double inv[3] = { 1.0 / d.x, 1.0 / d.y, 1.0 / d.z };
    double oo[3] = { o.x, o.y, o.z };
    for (int k = 0; k < S->num_pair; k++) {
        if (S->pair_bbox) {
            /* world box cull in double: skip pairs the ray cannot reach before the best hit */
            const float* bb = S->pair_bbox + 6 * k;
            double t0 = tmin, t1 = best;
            for (int a = 0; a < 3; a++) {
                double ta = (bb[a] - oo[a]) * inv[a], tb = (bb[3 + a] - oo[a]) * inv[a];
                if (ta > tb) { double t = ta; ta = tb; tb = t; }
                if (ta == ta && ta > t0) t0 = ta;
                if (tb == tb && tb < t1) t1 = tb;
            }
            if (t0 > t1) continue;
        }
        const float* m = S->inst_inv + 16 * S->pair_inst[k];
        vec_f lo = rowx_f(m, mk_f(o.x, o.y, o.z), 1.f), ld = rowx_f(m, mk_f(d.x, d.y, d.z), 0.f);
        float is[4];
        /* OptiX ignores a report outside [tmin, tmax]: a convexpolyhedron wholly behind the ray
           reports valid with t = 0 (CSG/csg_intersect_leaf_convexpolyhedron.h:85-101) */
        if (prim_f(is, &g, S->pair_node[k], tmin, lo, ld, err) && is[3] >= tmin && is[3] < best) {
            best = is[3]; bi = k;
            memcpy(bis, is, sizeof(bis));
            float lx = lo.x + is[3] * ld.x, ly = lo.y + is[3] * ld.y, lz = lo.z + is[3] * ld.z;
            blc = lz / sqrtf(lx * lx + ly * ly + lz * lz);
        }
    }
    if (bi < 0) { prd->gpbd = 0xffffffffu; return 0; }
    const float* m = S->inst_inv + 16 * S->pair_inst[bi];
    vec_f n = colx_f(m, mk_f(bis[0], bis[1], bis[2]), 0.f);
    prd->n = V(n.x, n.y, n.z);
    prd->t = best;
    prd->lposcost = blc;
    prd->gpbd = S->pair_gpbd[bi];
    prd->iiid = S->pair_iiid[bi];
    return 1;
}

/* ------------------------------------------------------------------ propagation */
enum { CONTINUE = 0, BREAK = 1, BOUNDARY = 2 };

typedef struct { f4 m1, m1g, m2, su; unsigned opt[4]; unsigned m1idx, m2idx; } state_t;

/* FP64 score accumulator of the adjoint estimator (same terms as the engine's, in double):
 * d log p / d theta for 8 wavelength bins x (absorption length, Rayleigh length, reemission
 * probability, refractive index) of material `mat` (1-based index), weights = the linear texture
 * interpolation weights of the 1 nm samples falling in each bin. */
typedef struct { double g[32]; unsigned mat; double nm0, nms, wl_lo, binw; } oscore;

static void oscore_add(oscore* S, int kind, float wl, double v)
{
    double fx = ((double)wl - S->nm0) / S->nms, f = floor(fx), a = fx - f;
    double l0 = S->nm0 + f * S->nms, l1 = l0 + S->nms;
    int b0 = (int)floor((l0 - S->wl_lo) / S->binw), b1 = (int)floor((l1 - S->wl_lo) / S->binw);
    if (b0 >= 0 && b0 < 8) S->g[kind * 8 + b0] += (1.0 - a) * v;
    if (b1 >= 0 && b1 < 8) S->g[kind * 8 + b1] += a * v;
}

/* TransCoeff and its derivatives in n1, n2 (analytic, double) */
static double trans_T(double n1, double n2, double c1, double ex, double ey)
{
    double eta = n1 / n2, c2 = sqrt(1.0 - eta * eta * (1.0 - c1 * c1));
    double n1c1 = n1 * c1, n2c2 = n2 * c2, n2c1 = n2 * c1, n1c2 = n1 * c2;
    double tx = 2.0 * n1c1 * ex / (n1c1 + n2c2), ty = 2.0 * n1c1 * ey / (n2c1 + n1c2);
    return n2c2 * (tx * tx + ty * ty) / n1c1;
}

static void rayleigh(photon_t* p, ustream* r)
{
    v3 dir, pol;
    int looping;
    do {
        float u0 = U(r), u1 = U(r), u2 = U(r), u3 = U(r), u4 = U(r);
        float ct = u0, st = sqrtf(1.0f - u0 * u0);
        if (u1 < 0.5f) ct = -ct;
        float sp = sinf(2.f * PI_F * u2), cp = cosf(2.f * PI_F * u2);
        dir = V(st * cp, st * sp, ct);
        rotate_uz(&dir, p->mom);
        float c = -dot3(dir, p->pol);
        pol = V(p->pol.x + c * dir.x, p->pol.y + c * dir.y, p->pol.z + c * dir.z);
        if (dot3(pol, pol) == 0.f) {
            sp = sinf(2.f * PI_F * u3); cp = cosf(2.f * PI_F * u3);
            pol = V(cp, sp, 0.f);
            rotate_uz(&pol, dir);
        } else if (u3 < 0.5f) pol = mul(-1.f, pol);
        pol = norm3(pol);
        float dc = dot3(pol, p->pol);
        looping = dc * dc < u4;
    } while (looping && !r->over);
    p->mom = dir;
    p->pol = pol;
}

static int to_boundary(unsigned* flag, photon_t* p, ustream* r, const state_t* s, float dist, const oracle_scene* S, oscore* sc)
{
    float ul = s->m1.y, sl = s->m1.z, rp = s->m1.w, gv = s->m1g.x;
    float us = U(r), ua = U(r);
    float sd = -sl * logf(us), ad = -ul * logf(ua);
    int scored = sc && s->m1idx == sc->mat;
    double La = ul, Ls = sl;
    if (ad <= sd) {
        if (ad <= dist) {
            p->time += ad / gv;
            p->pos = add(p->pos, mul(ad, p->mom));
            float ur = rp == 0.f ? 2.f : U(r);
            if (scored) {
                oscore_add(sc, 0, p->wavelength, -1.0 / La + (double)ad / (La * La));
                oscore_add(sc, 1, p->wavelength, (double)ad / (Ls * Ls));
                oscore_add(sc, 2, p->wavelength, ur < rp ? 1.0 / rp : -1.0 / (1.0 - rp));
            }
            if (ur < rp) {
                float uw = U(r), a = U(r), b = U(r), c = U(r), d = U(r);
                p->wavelength = scint_wl(S, uw);
                p->mom = uniform_sphere(a, b);
                p->pol = norm3(cross3(uniform_sphere(c, d), p->mom));
                *flag = 0x10;
                return CONTINUE;
            }
            *flag = 0x8;
            return BREAK;
        }
    } else if (sd <= dist) {
        if (scored) {
            oscore_add(sc, 1, p->wavelength, -1.0 / Ls + (double)sd / (Ls * Ls));
            oscore_add(sc, 0, p->wavelength, (double)sd / (La * La));
        }
        p->time += sd / gv;
        p->pos = add(p->pos, mul(sd, p->mom));
        rayleigh(p, r);
        *flag = 0x20;
        return CONTINUE;
    }
    if (scored) {
        oscore_add(sc, 0, p->wavelength, (double)dist / (La * La));
        oscore_add(sc, 1, p->wavelength, (double)dist / (Ls * Ls));
    }
    p->pos = add(p->pos, mul(dist, p->mom));
    p->time += dist / gv;
    return BOUNDARY;
}

static int at_boundary(unsigned* flag, photon_t* p, ustream* r, const state_t* s, v3 nrm, oscore* sc)
{
    float n1 = s->m1.x, n2 = s->m2.x, eta = n1 / n2;
    float _c1 = -dot3(p->mom, nrm);
    v3 on = _c1 < 0.f ? mul(-1.f, nrm) : nrm;
    v3 tr = cross3(p->mom, on);
    float tl = len3(tr);
    int ni = tl < 1e-6f;
    v3 At = ni ? p->pol : mul(1.0f / tl, tr);
    float Ep = dot3(p->pol, At);
    float c1 = fabsf(_c1);
    float c2c2 = 1.f - eta * eta * (1.f - c1 * c1);
    int tir = c2c2 < 0.f;
    float EdotN = dot3(p->pol, on);
    float c2 = tir ? 0.f : sqrtf(c2c2);
    float n1c1 = n1 * c1, n2c2 = n2 * c2, n2c1 = n2 * c1, n1c2 = n1 * c2;
    float E1x = ni ? 0.f : Ep, E1y = ni ? 1.f : len3(sub(p->pol, mul(Ep, At)));
    float Etx = 2.f * n1c1 * E1x / (n1c1 + n2c2), Ety = 2.f * n1c1 * E1y / (n2c1 + n1c2);
    float Erx = Etx - E1x, Ery = (n2 * Ety / n1) - E1y;
    float ir = 1.0f / sqrtf(Erx * Erx + Ery * Ery), it = 1.0f / sqrtf(Etx * Etx + Ety * Ety);
    float RRx = Erx * ir, RRy = Ery * ir, TTx = Etx * it, TTy = Ety * it;
    float T = (tir || n1c1 == 0.f) ? 0.f : n2c2 * (Etx * Etx + Ety * Ety) / n1c1;
    float u = U(r);
    int refl = u > T;
    if (sc && !tir && n1c1 != 0.f && T > 0.f && T < 1.f && (s->m1idx == sc->mat || s->m2idx == sc->mat)) {
        double k = refl ? -1.0 / (1.0 - (double)T) : 1.0 / (double)T;
        double h1 = 1e-6 * n1, h2 = 1e-6 * n2;
        /* central differences of the analytic T in double (step 1e-6 relative) */
        if (s->m1idx == sc->mat)
            oscore_add(sc, 3, p->wavelength, k * (trans_T(n1 + h1, n2, c1, E1x, E1y) - trans_T(n1 - h1, n2, c1, E1x, E1y)) / (2 * h1));
        if (s->m2idx == sc->mat)
            oscore_add(sc, 3, p->wavelength, k * (trans_T(n1, n2 + h2, c1, E1x, E1y) - trans_T(n1, n2 - h2, c1, E1x, E1y)) / (2 * h2));
    }
    p->mom = refl ? add(p->mom, mul(2.0f * c1, on)) : add(mul(eta, p->mom), mul(eta * c1 - c2, on));
    v3 Ap = norm3(cross3(p->mom, At));
    if (ni) p->pol = refl ? mul(n2 > n1 ? -1.f : 1.f, p->pol) : p->pol;
    else if (refl) p->pol = tir ? add(mul(-1.f, p->pol), mul(2.f * EdotN, on)) : add(mul(RRx, At), mul(RRy, Ap));
    else p->pol = add(mul(TTx, At), mul(TTy, Ap));
    *flag = refl ? 0x400 : 0x800;
    return CONTINUE;
}

static void marsaglia(v3* dir, ustream* r)
{
    float u, v, b;
    do { u = 2.f * U(r) - 1.f; v = 2.f * U(r) - 1.f; b = u * u + v * v; } while (b > 1.f && !r->over);
    float a = 2.f * sqrtf(1.f - b);
    *dir = V(a * u, a * v, 2.f * b - 1.f);
}

static int at_surface(unsigned* flag, photon_t* p, ustream* r, const state_t* s, v3 nrm)
{
    float det = s->su.x, abs_ = s->su.y, rd = s->su.w;
    float u = U(r);
    if (u < abs_ + det) { *flag = u < abs_ ? 0x80 : 0x40; return BREAK; }
    if (u < abs_ + det + rd) {
        *flag = 0x100;
        v3 old = p->mom;
        float orient = dot3(old, nrm) > 0.f ? -1.f : 1.f;
        float ndv, uu;
        int count = 0;
        do {
            count++;
            marsaglia(&p->mom, r);
            ndv = dot3(p->mom, nrm) * orient;
            if (ndv < 0.f) { p->mom = mul(-1.f, p->mom); ndv = -ndv; }
            uu = U(r);
        } while (!(uu < ndv) && count < 1024 && !r->over);
        v3 fn = norm3(sub(p->mom, old));
        float e = dot3(p->pol, fn);
        p->pol = add(mul(-1.f, p->pol), mul(2.f * e, fn));
    } else {
        *flag = 0x200;
        float pn = dot3(p->mom, nrm);
        p->mom = sub(p->mom, mul(2.f * pn, nrm));
        float e = dot3(p->pol, nrm);
        p->pol = add(mul(-1.f, p->pol), mul(2.f * e, nrm));
    }
    return CONTINUE;
}

static int propagate(photon_t* p, ustream* r, const prd_t* prd, const oracle_scene* S, oscore* sc)
{
    unsigned bnd = prd->gpbd & 0xffffu, id = prd->iiid & 0xffffu, ii = prd->iiid >> 16;
    v3 n = prd->n;
    float ct = dot3(p->mom, n);
    p->obf = (p->obf & 0x8000ffffu) | ((bnd & 0x7fffu) << 16);
    p->identity = (p->identity & 0xff000000u) | (id & 0xffffffu);
    p->obf = (p->obf & 0x7fffffffu) | ((ct < 0.f ? 1u : 0u) << 31);
    p->hitcount_iindex = 0x10000u | (ii & 0xffffu);
    int line = (int)bnd * 4;
    int m1 = ct > 0.f ? line + 3 : line, m2 = ct > 0.f ? line : line + 3, su = ct > 0.f ? line + 2 : line + 1;
    state_t s;
    s.m1 = bnd_lookup(S, p->wavelength, m1, 0);
    s.m1g = bnd_lookup(S, p->wavelength, m1, 1);
    s.m2 = bnd_lookup(S, p->wavelength, m2, 0);
    s.su = bnd_lookup(S, p->wavelength, su, 0);
    memcpy(s.opt, S->optical + 4 * su, 16);
    s.m1idx = S->optical[4 * m1];
    s.m2idx = S->optical[4 * m2];
    unsigned flag = 0;
    int cmd = to_boundary(&flag, p, r, &s, prd->t, S, sc);
    if (cmd == BOUNDARY) {
        int ems = (int)s.opt[1];
        if (ems == 1) cmd = at_boundary(&flag, p, r, &s, n, sc);
        else if (ems == 2) cmd = at_surface(&flag, p, r, &s, n);
        else if (prd->lposcost < 0.f) cmd = at_surface(&flag, p, r, &s, n);
        else if (ems == 3) { (void)U(r); flag = 0x40; cmd = BREAK; }
    }
    set_flag(p, flag);
    return cmd;
}

static void add_nibble(uint64_t* his, uint64_t* bnd, unsigned slot, unsigned flag, unsigned boundary)
{
    unsigned iseq = slot / 16, shift = 4 * (slot - iseq * 16);
    if (iseq < 2) {
        unsigned ffs = 0;
        for (unsigned b = 0; b < 32; b++) if (flag & (1u << b)) { ffs = b + 1; break; }
        his[iseq] |= ((uint64_t)(ffs & 0xf)) << shift;
        bnd[iseq] |= ((uint64_t)(boundary & 0xf)) << shift;
    }
}

/* photon loop.  gs (G,6,4); uniforms (n,K) for photons first..first+n-1 of the event;
 * photon out (n,4,4) float; seq out (n,4) u64 ; returns OR of error bits:
 *   1 CSG evaluator error, 2 uniform stream exhausted */
static int run_photons(const oracle_scene* S, const float* gs, int G, long long first, long long n,
                       const float* uniforms, int K, float* photon, uint64_t* seq,
                       const oscore* proto, int num_sensor, double* hits, double* grad);

int oracle_simulate(const oracle_scene* S, const float* gs, int G, long long first, long long n,
                    const float* uniforms, int K, float* photon, uint64_t* seq)
{
    return run_photons(S, gs, G, first, n, uniforms, K, photon, seq, NULL, 0, NULL, NULL);
}

/* FP64 reference of the adjoint estimator: hits[s] and grad[s*32+k] = sum over hits on sensor s
 * of the path score, with the same photons as oracle_simulate (scene tables already re-tabulated) */
int oracle_adjoint(const oracle_scene* S, const float* gs, int G, long long first, long long n, const float* uniforms, int K,
                   unsigned mat, double nm0, double nms, double wl_lo, double binw, int num_sensor, double* hits, double* grad)
{
    oscore proto;
    memset(&proto, 0, sizeof(proto));
    proto.mat = mat; proto.nm0 = nm0; proto.nms = nms; proto.wl_lo = wl_lo; proto.binw = binw;
    return run_photons(S, gs, G, first, n, uniforms, K, NULL, NULL, &proto, num_sensor, hits, grad);
}

static int run_photons(const oracle_scene* S, const float* gs, int G, long long first, long long n,
                       const float* uniforms, int K, float* photon, uint64_t* seq,
                       const oscore* proto, int num_sensor, double* hits, double* grad)
{
    long long* off = (long long*)malloc(sizeof(long long) * (G + 1));
    off[0] = 0;
    for (int g = 0; g < G; g++) { int32_t c; memcpy(&c, gs + 24 * g + 3, 4); off[g + 1] = off[g] + (c > 0 ? c : 0); }
    int err_all = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : err_all)
    for (long long j = 0; j < n; j++) {
        long long idx = first + j;
        int gi = 0;
        while (gi + 1 < G && off[gi + 1] <= idx) gi++;
        const float* g = gs + 24 * gi;
        ustream r = { uniforms + (size_t)j * K, K, 0, 0 };
        photon_t p;
        memset(&p, 0, sizeof(p));
        int32_t code;
        memcpy(&code, g, 4);
        if (code == 6) {
            gen_torch(&p, &r, g, (unsigned long long)idx);
            /* qudarap/qsim.h:2541-2544: no wavelength given, a black-body one (qplanck::wavelength) */
            if (p.wavelength <= 0.f && S->planck) { float u = U(&r); p.wavelength = tex2d_f1(S->planck, 4096, 1, u, 0.5f); }
        }
        else if (code == 16 || code == 5) gen_scint(&p, &r, g, S);
        else if (code == 15 || code == 18) gen_cerenkov(&p, &r, g, S);
        else if (code == 14) gen_carrier(&p, g, (unsigned long long)idx);
        else if (code == 19) {
            /* qudarap/qsim.h:2557: the input photon as given, TORCH flag set */
            if (S->input_photon && idx < S->num_input) memcpy(&p, S->input_photon + 16 * (size_t)idx, sizeof(p));
            set_flag(&p, 0x4);
        }
        p.index = (unsigned)(idx & 0xffffffffu);
        p.identity = ((unsigned)((idx >> 32) & 0xff) << 24) | (p.identity & 0xffffffu);
        uint64_t his[2] = { 0, 0 }, bn[2] = { 0, 0 };
        int err = 0;
        oscore score, *sc = NULL;
        if (proto) { score = *proto; memset(score.g, 0, sizeof(score.g)); sc = &score; }
        add_nibble(his, bn, 0, p.obf & 0xffffu, (p.obf >> 16) & 0x7fffu);
        int bounce = 0;
        while (bounce < S->max_bounce && p.time < S->max_time) {
            float tmin = (p.obf & S->eps0_mask) ? S->tmin0 : S->tmin;
            prd_t prd;
            memset(&prd, 0, sizeof(prd));
            trace(S, p.pos, p.mom, tmin, &prd, &err);
            if ((prd.gpbd & 0xffffu) == 0xffffu) break;
            prd.n = norm3(prd.n);
            int cmd = propagate(&p, &r, &prd, S, sc);
            bounce++;
            add_nibble(his, bn, (unsigned)bounce, p.obf & 0xffffu, (p.obf >> 16) & 0x7fffu);
            if (cmd == BREAK) break;
        }
        if (sc && (p.flagmask & S->hit_mask) == S->hit_mask) {
            unsigned id = p.identity & 0xffffffu;
            if (id > 0 && (int)(id - 1) < num_sensor) {
#pragma omp critical
                {
                    hits[id - 1] += 1.0;
                    for (int k = 0; k < 32; k++) grad[(size_t)(id - 1) * 32 + k] += sc->g[k];
                }
            }
        }
        if (!photon) { err_all |= (err ? 1 : 0) | (r.over ? 2 : 0); continue; }
        float* o = photon + 16 * j;
        o[0] = p.pos.x; o[1] = p.pos.y; o[2] = p.pos.z; o[3] = p.time;
        o[4] = p.mom.x; o[5] = p.mom.y; o[6] = p.mom.z; memcpy(o + 7, &p.hitcount_iindex, 4);
        o[8] = p.pol.x; o[9] = p.pol.y; o[10] = p.pol.z; o[11] = p.wavelength;
        memcpy(o + 12, &p.obf, 4); memcpy(o + 13, &p.identity, 4); memcpy(o + 14, &p.index, 4); memcpy(o + 15, &p.flagmask, 4);
        if (seq) { seq[4 * j + 0] = his[0]; seq[4 * j + 1] = his[1]; seq[4 * j + 2] = bn[0]; seq[4 * j + 3] = bn[1]; }
        err_all |= (err ? 1 : 0) | (r.over ? 2 : 0);
    }
    free(off);
    return err_all;
}

/* texture emulation exposed for the hardware-filtering pin test */
float oracle_tex2d_f1(const float* data, int W, int H, float x, float y) { return tex2d_f1(data, W, H, x, y); }
void oracle_tex2d_f4(const float* data, int W, int H, float x, float y, float* out)
{
    f4 r = tex2d_f4(data, W, H, x, y);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

int oracle_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
