// phx_physics.cuh : optical photon generation and one-bounce propagation physics.
//
// Each function restates the reference's device physics with the same random-number
// consumption order and the same float operation order (bit-exact seqhis is the target):
//   uniform_sphere          qudarap/qsim.h:180-201
//   lambertian_direction    qudarap/qsim.h:433-486
//   random_direction_marsaglia qudarap/qsim.h:554-575
//   rayleigh_scatter        qudarap/qsim.h:604-692
//   propagate_to_boundary   qudarap/qsim.h:721-866
//   propagate_at_boundary   qudarap/qsim.h:1001-1208
//   propagate_at_surface    qudarap/qsim.h:1680-1758
//   reflect_diffuse/specular qudarap/qsim.h:1988-2093
//   propagate (dispatch)    qudarap/qsim.h:2229-2338
//   fill_state              qudarap/qbnd.h:108-224
//   torch generation        sysrap/storch.h:192-520
//   scintillation           qudarap/qscint.h:66-157, 251-258
//   Cerenkov                qudarap/qcerenkov.h:56-137, 285-320
// Random numbers are cuRAND XORWOW (called through curand_kernel.h, not reimplemented).
#pragma once
#include <curand_kernel.h>
#include "phx_vec.cuh"
#include "phx_pod.h"
#include "phx_csg.cuh"

enum { PHX_CONTINUE = 0, PHX_BREAK = 1, PHX_BOUNDARY = 2 };

struct PhxPhoton {
    float3 pos; float time;
    float3 mom; unsigned hitcount_iindex;
    float3 pol; float wavelength;
    unsigned obf; unsigned identity; unsigned index; unsigned flagmask;

    PHX_D unsigned flag() const { return obf & 0xffffu; }
    PHX_D unsigned boundary() const { return (obf & 0x7fff0000u) >> 16; }
    PHX_D void set_flag(unsigned f) { obf = (obf & 0xffff0000u) | (f & 0xffffu); flagmask |= f; }
    PHX_D void zero_flags() { obf = 0u; identity = 0u; index = 0u; flagmask = 0u; hitcount_iindex = 0u; }
    PHX_D void set_index(unsigned long long full)
    {
        index = (unsigned)(full & 0xffffffffull);
        identity = ((unsigned)((full >> 32) & 0xffull) << 24) | (identity & 0xffffffu);
    }
    // sphoton::set_prd  sysrap/sphoton.h:499-505
    PHX_D void set_prd(unsigned bnd, unsigned id, float orient, unsigned ii)
    {
        obf = (obf & 0x8000ffffu) | ((bnd & 0x7fffu) << 16);
        identity = (identity & 0xff000000u) | (id & 0x00ffffffu);
        obf = (obf & 0x7fffffffu) | ((orient < 0.f ? 0x1u : 0x0u) << 31);
        hitcount_iindex = 0x00010000u | (0x0000ffffu & ii);
    }
};

// per-ray data returned by the closest-hit search (quad2 layout sysrap/squad.h:180-245)
struct PhxPRD {
    float3 normal; float distance;
    float lposcost; unsigned ii_id; unsigned gp_bd;
    PHX_D unsigned boundary() const { return gp_bd & 0xffffu; }
    PHX_D unsigned identity() const { return ii_id & 0xffffu; }
    PHX_D unsigned iindex() const { return ii_id >> 16; }
};

struct PhxState {
    float4 material1;   // rindex, absorption length, scattering length, reemission prob
    float4 m1group2;    // group velocity
    float4 material2;
    float4 surface;     // detect, absorb, reflect specular, reflect diffuse
    uint4 optical;      // x: 1-based surface index (0: none) ; y: ems
    unsigned m1idx, m2idx;   // 1-based material indices of m1/m2 (qbnd s.index.x/y; adjoint only)
};

// Score-function accumulator of the adjoint: d log p(path) / d theta for the properties of one
// material tabulated in 8 wavelength bins (kind 0 absorption length, 1 Rayleigh length,
// 2 reemission probability, 3 refractive index).  A property at wavelength wl is the texture's
// linear interpolation of its 1 nm samples, so d prop / d theta_b is the filter weight of the
// samples that lie in bin b.
//
// The refractive index also moves the path itself: a refracted direction depends on n, so every
// later segment length, incidence angle and Fresnel probability does.  With the path's random
// variables held fixed (event distances, branch choices, sampled directions), that pathwise part
// of d log p / d n is carried forward as a tangent: the derivatives of the position, direction and
// polarisation with respect to nu, the parametrised index at the photon's current wavelength.
// A hit point's tangent and the change of the surface normal come from a probe: the same prim
// intersected along the ray moved a small step along the tangent.
// The 32 score terms of a path live in shared memory, term-major with one word per thread of the
// block (term k of thread t at word k * PHX_SCORE_LANES + t: a warp's accesses to one term hit 32
// banks), not in the thread's local memory: they are indexed by wavelength bin at run time, and as
// local memory (128 B of a 1.4 KB stack frame per thread, over 56k resident threads) every update
// missed L1.  Kernels that carry scores run blocks of at most PHX_SCORE_LANES threads.
#define PHX_SCORE_LANES 128
#define PHX_SG(S, k) ((S).g[(k) * PHX_SCORE_LANES])
struct PhxScore {
    float* g;                  // this thread's first term in the block's shared score area
    unsigned mat;              // 1-based material index of the parametrised material
    float nm0, nms;            // texture wavelength domain
    float wl_lo, binw;         // bins [wl_lo + b binw, wl_lo + (b+1) binw), b < 8
    float3 tpos, tdir, tpol;   // d pos, d mom, d pol / d nu
    int pathwise;              // carry the tangent (0: score terms only)
    PhxCsgCtx csg;             // geometry of the probe intersections
    const float4* inst_inv;
    const int* prim_node;      // root node of each prim (globalPrimIdx)
    float tmin, tmin0;         // the trace's tmin by the last flag (probe intersections use the same)
    unsigned eps0_mask;
};

PHX_D void score_tangent_reset(PhxScore& S)
{
    S.tpos = make_float3(0.f, 0.f, 0.f);
    S.tdir = S.tpos;
    S.tpol = S.tpos;
}

PHX_D bool score_tangent_zero(const PhxScore& S)
{
    return S.tpos.x == 0.f && S.tpos.y == 0.f && S.tpos.z == 0.f && S.tdir.x == 0.f && S.tdir.y == 0.f && S.tdir.z == 0.f &&
           S.tpol.x == 0.f && S.tpol.y == 0.f && S.tpol.z == 0.f;
}

PHX_D void score_add(PhxScore& S, int kind, float wl, float v)
{
    const float fx = (wl - S.nm0) / S.nms;
    const float f = floorf(fx);
    const float a = fx - f;
    const float l0 = S.nm0 + f * S.nms, l1 = l0 + S.nms;
    const int b0 = (int)floorf((l0 - S.wl_lo) / S.binw);
    const int b1 = (int)floorf((l1 - S.wl_lo) / S.binw);
    if (b0 >= 0 && b0 < 8) PHX_SG(S, kind * 8 + b0) += (1.f - a) * v;
    if (b1 >= 0 && b1 < 8) PHX_SG(S, kind * 8 + b1) += a * v;
}

// a refractive-index term of the path: clipped at PHX_ADJ_SCORE_CAP (terms near the critical angle, at
// grazing incidence and along the dipole axis of a scattering have a finite mean and no finite
// variance).  The two caps were chosen against central differences on the detector's 1M-photon
// event: 1e3 / 10 leave the dominant bins 6-18 % low, 1e4 / 100 within the differences' 2-6 %
// errors, 1e5 lets single photons dominate the sum again.
#ifndef PHX_ADJ_SCORE_CAP
#define PHX_ADJ_SCORE_CAP 10000.f
#endif
PHX_D void score_add_capped(PhxScore& S, float wl, float v)
{
    score_add(S, 3, wl, fminf(fmaxf(v, -PHX_ADJ_SCORE_CAP), PHX_ADJ_SCORE_CAP));
}

// forward-mode dual numbers for d TransCoeff / d n
struct PhxDual { float v, d; };
PHX_D PhxDual dd(float v, float d) { PhxDual r; r.v = v; r.d = d; return r; }
PHX_D PhxDual operator+(PhxDual a, PhxDual b) { return dd(a.v + b.v, a.d + b.d); }
PHX_D PhxDual operator-(PhxDual a, PhxDual b) { return dd(a.v - b.v, a.d - b.d); }
PHX_D PhxDual operator*(PhxDual a, PhxDual b) { return dd(a.v * b.v, a.d * b.v + a.v * b.d); }
PHX_D PhxDual operator/(PhxDual a, PhxDual b) { return dd(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
PHX_D PhxDual dsqrt(PhxDual a) { const float r = sqrtf(a.v); return dd(r, r > 0.f ? 0.5f * a.d / r : 0.f); }

PHX_D PhxDual operator-(PhxDual a) { return dd(-a.v, -a.d); }
PHX_D PhxDual dfabs(PhxDual a) { return a.v < 0.f ? -a : a; }

// dual 3-vectors: value and tangent
struct PhxDual3 { float3 v, d; };
PHX_D PhxDual3 d3(float3 v, float3 d) { PhxDual3 r; r.v = v; r.d = d; return r; }
PHX_D PhxDual3 operator+(PhxDual3 a, PhxDual3 b) { return d3(a.v + b.v, a.d + b.d); }
PHX_D PhxDual3 operator-(PhxDual3 a, PhxDual3 b) { return d3(a.v - b.v, a.d - b.d); }
PHX_D PhxDual3 operator*(PhxDual s, PhxDual3 a) { return d3(s.v * a.v, s.d * a.v + s.v * a.d); }
PHX_D PhxDual ddot(PhxDual3 a, PhxDual3 b) { return dd(dot(a.v, b.v), dot(a.d, b.v) + dot(a.v, b.d)); }
PHX_D PhxDual3 dcross(PhxDual3 a, PhxDual3 b) { return d3(cross(a.v, b.v), cross(a.d, b.v) + cross(a.v, b.d)); }
PHX_D PhxDual3 dnormalize(PhxDual3 a)
{
    const PhxDual l = dsqrt(ddot(a, a));
    const PhxDual inv = dd(1.f, 0.f) / l;
    return inv * a;
}

// TransCoeff of propagate_at_boundary as a function of (n1, n2) at fixed c1 and E1 amplitudes
PHX_D PhxDual trans_coeff_dual(PhxDual n1, PhxDual n2, float c1, float E1x, float E1y)
{
    const PhxDual one = dd(1.f, 0.f), two = dd(2.f, 0.f), C1 = dd(c1, 0.f);
    const PhxDual eta = n1 / n2;
    const PhxDual c2 = dsqrt(one - eta * eta * (one - C1 * C1));
    const PhxDual n1c1 = n1 * C1, n2c2 = n2 * c2, n2c1 = n2 * C1, n1c2 = n1 * c2;
    const PhxDual tx = two * n1c1 * dd(E1x, 0.f) / (n1c1 + n2c2);
    const PhxDual ty = two * n1c1 * dd(E1y, 0.f) / (n2c1 + n1c2);
    return n2c2 * (tx * tx + ty * ty) / n1c1;
}

struct PhxProps {
    cudaTextureObject_t bnd_tex;    // (num_wl) x (num_bnd*4*2) float4, linear, normalized, wrap
    const uint4* optical;           // (num_bnd*4)
    float nm0, nms;                 // wavelength domain low and step (nm)
    unsigned nx, ny;                // texture width/height
    cudaTextureObject_t icdf_tex;   // 4096 x 3 float, linear, normalized, wrap
    unsigned hd_factor;
    cudaTextureObject_t planck_tex; // PHX_PLANCK_N x 1 float black-body wavelength ICDF, linear, normalized, wrap
    const float4* input_photon;     // (num_input_photon*4) sphoton rows for INPUT_PHOTON gensteps, or null
    long long num_input_photon;
};

PHX_D float phx_uniform(curandStateXORWOW& r) { return curand_uniform(&r); }

PHX_D float4 boundary_lookup(const PhxProps& P, float nm, unsigned line, unsigned k)
{
    float fx = (nm - P.nm0) / P.nms;
    float x = (fx + 0.5f) / float(P.nx);
    unsigned iy = 2u * line + k;
    float y = (float(iy) + 0.5f) / float(P.ny);
    return tex2D<float4>(P.bnd_tex, x, y);
}

template <bool ADJ = false>
PHX_D void fill_state(PhxState& s, const PhxProps& P, unsigned boundary, float wavelength, float cosTheta)
{
    const int line = boundary * 4;
    const int m1_line = cosTheta > 0.f ? line + 3 : line + 0;
    const int m2_line = cosTheta > 0.f ? line + 0 : line + 3;
    const int su_line = cosTheta > 0.f ? line + 2 : line + 1;
    s.material1 = boundary_lookup(P, wavelength, m1_line, 0);
    s.m1group2 = boundary_lookup(P, wavelength, m1_line, 1);
    s.material2 = boundary_lookup(P, wavelength, m2_line, 0);
    s.surface = boundary_lookup(P, wavelength, su_line, 0);
    s.optical = __ldg(P.optical + su_line);
    if (ADJ) {
        s.m1idx = __ldg(&P.optical[m1_line].x);
        s.m2idx = __ldg(&P.optical[m2_line].x);
    }
}

// hd20 inverse-CDF lookup qudarap/qscint.h:251-258 (hd10/hd0 for other tables)
PHX_D float scint_wavelength(const PhxProps& P, float u0)
{
    if (P.hd_factor == 20u) {
        const bool is_lhs = (u0 < 0.05f);
        const bool is_rhs = (u0 > 0.95f);
        const float x = is_lhs ? (u0 * 20.f) : (is_rhs ? (u0 - 0.95f) * 20.f : u0);
        const float y = is_lhs ? 1.5f / 3.f : (is_rhs ? 2.5f / 3.f : 0.5f / 3.f);
        return tex2D<float>(P.icdf_tex, x, y);
    } else if (P.hd_factor == 10u) {
        const bool is_lhs = (u0 < 0.1f);
        const bool is_rhs = (u0 > 0.9f);
        const float x = is_lhs ? (u0 * 10.f) : (is_rhs ? (u0 - 0.9f) * 10.f : u0);
        const float y = is_lhs ? 1.5f / 3.f : (is_rhs ? 2.5f / 3.f : 0.5f / 3.f);
        return tex2D<float>(P.icdf_tex, x, y);
    } else if (P.hd_factor == 0u) {
        return tex2D<float>(P.icdf_tex, u0, 0.5f / 3.f);
    }
    return 0.f;
}

PHX_D float3 uniform_sphere(float u0, float u1)
{
    float phi = u0 * 2.f * PHX_PI_F;
    float cosTheta = 2.f * u1 - 1.f;
    float sinTheta = sqrtf(1.f - cosTheta * cosTheta);
    return make_float3(cosf(phi) * sinTheta, sinf(phi) * sinTheta, cosTheta);
}

// ---------------------------------------------------------------- generation
// quad6 genstep access: g[0..5] float4 rows
PHX_D void generate_torch(PhxPhoton& p, curandStateXORWOW& rng, const float4* g, unsigned long long photon_id)
{
    const float4 q1 = g[1], q2 = g[2], q3 = g[3], q4 = g[4], q5 = g[5];
    const unsigned numphoton = __float_as_uint(g[0].w);
    const float3 gpos = make_float3(q1.x, q1.y, q1.z);
    const float gtime = q1.w;
    const float3 gmom = make_float3(q2.x, q2.y, q2.z);
    const float gwl = q3.w;
    const float2 zenith = make_float2(q4.x, q4.y);
    const float2 azimuth = make_float2(q4.z, q4.w);
    const float radius_ = q5.x;
    const float distance = q5.y;
    const unsigned type = __float_as_uint(q5.w);

    if (type == PHX_T_DISC) {
        p.wavelength = gwl; p.time = gtime; p.mom = gmom;
        float u_zenith = zenith.x + phx_uniform(rng) * (zenith.y - zenith.x);
        float u_azimuth = azimuth.x + phx_uniform(rng) * (azimuth.y - azimuth.x);
        float r = radius_ * u_zenith;
        float phi = 2.f * PHX_PI_F * u_azimuth;
        float sinPhi = sinf(phi), cosPhi = cosf(phi);
        p.pos = make_float3(r * cosPhi, r * sinPhi, 0.f);
        rotate_uz(p.pos, p.mom);
        p.pos = p.pos + gpos;
        p.pol = make_float3(sinPhi, -cosPhi, 0.f);
        rotate_uz(p.pol, p.mom);
    } else if (type == PHX_T_SPHERE || type == PHX_T_SPHERE_RANDPOL) {
        p.wavelength = gwl; p.time = gtime;
        float u_zenith = zenith.x + phx_uniform(rng) * (zenith.y - zenith.x);
        float u_azimuth = azimuth.x + phx_uniform(rng) * (azimuth.y - azimuth.x);
        float phi = 2.f * PHX_PI_F * u_azimuth;
        float sinPhi = sinf(phi), cosPhi = cosf(phi);
        float cosTheta = 1.f - 2.0f * u_zenith;
        float sinTheta = sqrtf(1.0f - cosTheta * cosTheta);
        float flip = copysignf(1.f, radius_);
        p.mom = make_float3(flip * sinTheta * cosPhi, flip * sinTheta * sinPhi, flip * cosTheta);
        float radius = fabsf(radius_);
        p.pos = make_float3(sinTheta * cosPhi * radius, sinTheta * sinPhi * radius, cosTheta * radius);
        float frac_twopi = type == PHX_T_SPHERE_RANDPOL ? phx_uniform(rng) : distance;
        float phase = 2.f * PHX_PI_F * frac_twopi;
        p.pol = make_float3(cosf(phase), sinf(phase), 0.f);
        rotate_uz(p.pol, p.mom);
    } else if (type == PHX_T_SPHERE_MARSAGLIA) {
        p.wavelength = gwl; p.time = gtime;
        float u0z, u1a, u, v, b, a;
        int count = 0;
        do {
            u0z = zenith.x + phx_uniform(rng) * (zenith.y - zenith.x);
            u1a = azimuth.x + phx_uniform(rng) * (azimuth.y - azimuth.x);
            u = 2.f * u0z - 1.f;
            v = 2.f * u1a - 1.f;
            b = u * u + v * v;
        } while (b > 1.f && ++count < 100000);
        a = 2.f * sqrtf(1.f - b);
        float radius = fabsf(radius_);
        float flip = copysignf(1.f, radius_);
        p.mom = make_float3(flip * a * u, flip * a * v, flip * (2.f * b - 1.f));
        p.pos = make_float3(a * u * radius, a * v * radius, (2.f * b - 1.f) * radius);
        float phase = 2.f * PHX_PI_F * distance;
        p.pol = make_float3(cosf(phase), sinf(phase), 0.f);
        rotate_uz(p.pol, p.mom);
    } else if (type == PHX_T_LINE) {
        p.wavelength = gwl; p.time = gtime; p.mom = gmom;
        float frac = float(photon_id) / float(numphoton);
        float sfrac = 2.f * (frac - 0.5f);
        float r = radius_ * sfrac;
        p.pos = make_float3(r, 0.f, 0.f);
        rotate_uz(p.pos, p.mom);
        p.pos = p.pos + gpos;
        p.pol = make_float3(0.f, -1.f, 0.f);
        rotate_uz(p.pol, p.mom);
    } else if (type == PHX_T_POINT) {
        p.wavelength = gwl; p.time = gtime; p.mom = gmom;
        p.pos = make_float3(0.f, 0.f, 0.f);
        rotate_uz(p.pos, p.mom);
        p.pos = p.pos + gpos;
        p.pol = make_float3(0.f, -1.f, 0.f);
        rotate_uz(p.pol, p.mom);
    } else if (type == PHX_T_CIRCLE) {
        p.wavelength = gwl; p.time = gtime;
        float f = float(photon_id) / float(numphoton);
        float frac = azimuth.x * (1.f - f) + azimuth.y * (f);
        float phi = 2.f * PHX_PI_F * frac;
        float sinPhi = sinf(phi), cosPhi = cosf(phi);
        float r = radius_ < 0.f ? -radius_ : radius_;
        p.mom = make_float3(radius_ < 0.f ? -cosPhi : cosPhi, 0.f, radius_ < 0.f ? -sinPhi : sinPhi);
        p.pos = make_float3(r * cosPhi, 0.f, r * sinPhi);
        p.pos = p.pos + gpos;
        p.pol = make_float3(0.f, -1.f, 0.f);
        rotate_uz(p.pol, p.mom);
    } else if (type == PHX_T_RECTANGLE) {
        p.wavelength = gwl; p.time = gtime;
        int side_size = (int)numphoton / 4;
        int side = (int)photon_id / side_size;
        int side_offset = side * side_size;
        int side_index = (int)photon_id - side_offset;
        float frac = float(side_index) / float(side_size);
        if (side == 0 || side == 1) {
            p.pos = make_float3(side == 0 ? azimuth.x : azimuth.y, 0.f, (1.f - frac) * zenith.x + frac * zenith.y);
            p.mom = make_float3(side == 0 ? 1.f : -1.f, 0.f, 0.f);
        } else if (side == 2 || side == 3) {
            p.pos = make_float3((1.f - frac) * azimuth.x + frac * azimuth.y, 0.f, side == 2 ? zenith.x : zenith.y);
            p.mom = make_float3(0.f, 0.f, side == 2 ? 1.f : -1.f);
        }
        p.pos = p.pos + gpos;
        p.pol = make_float3(0.f, -1.f, 0.f);
        rotate_uz(p.pol, p.mom);
    }
    p.zero_flags();
    p.set_flag(PHX_TORCH);
}

PHX_D void scint_mom_pol_wavelength(PhxPhoton& p, curandStateXORWOW& rng, const PhxProps& P)
{
    float u0 = phx_uniform(rng);
    float u1 = phx_uniform(rng);
    float u2 = phx_uniform(rng);
    float u3 = phx_uniform(rng);
    float cost = 1.f - 2.f * u0;
    float sint = sqrtf((1.f - cost) * (1.f + cost));
    float phi = 2.f * PHX_PI_F * u1;
    float sinp = sinf(phi);
    float cosp = cosf(phi);
    p.mom = make_float3(sint * cosp, sint * sinp, cost);
    p.pol = make_float3(cost * cosp, cost * sinp, -sint);
    phi = 2.f * PHX_PI_F * u2;
    sinp = sinf(phi);
    cosp = cosf(phi);
    p.pol = normalize(cosp * p.pol + sinp * cross(p.mom, p.pol));
    p.wavelength = scint_wavelength(P, u3);
}

PHX_D void generate_scint(PhxPhoton& p, curandStateXORWOW& rng, const float4* g, const PhxProps& P)
{
    scint_mom_pol_wavelength(p, rng, P);
    const float4 q1 = g[1], q2 = g[2], q3 = g[3], q5 = g[5];
    const float charge = q3.y;
    float fraction = charge == 0.f ? 1.f : phx_uniform(rng);
    p.pos = make_float3(q1.x, q1.y, q1.z) + fraction * make_float3(q2.x, q2.y, q2.z);
    float u4 = phx_uniform(rng);
    float deltaTime = fraction * q2.w / q3.w - q5.x * logf(u4);
    p.time = q1.w + deltaTime;
    p.zero_flags();
    p.set_flag(PHX_SCINTILLATION);
}

PHX_D void generate_cerenkov(PhxPhoton& p, curandStateXORWOW& rng, const float4* g, const PhxProps& P, unsigned& status)
{
    const float4 q0 = g[0], q1 = g[1], q2 = g[2], q3 = g[3], q4 = g[4], q5 = g[5];
    const unsigned matline = __float_as_uint(q0.z);
    const float3 dpos = make_float3(q2.x, q2.y, q2.z);
    const float step_length = q2.w;
    const float preVelocity = q3.w;
    const float BetaInverse = q4.x, Wmin = q4.y, Wmax = q4.z;
    const float maxSin2 = q5.x, Mean1 = q5.y, Mean2 = q5.z, postVelocity = q5.w;
    const float3 p0 = normalize(dpos);
    float wavelength, cosTheta, sin2Theta;
    {
        float u0, u1, w, sampledRI, u_maxSin2;
        unsigned count = 0;
        do {
            u0 = phx_uniform(rng);
            w = Wmin + u0 * (Wmax - Wmin);
            wavelength = Wmin * Wmax / w;
            float4 props = boundary_lookup(P, wavelength, matline, 0u);
            sampledRI = props.x;
            cosTheta = BetaInverse / sampledRI;
            sin2Theta = fmaxf(0.f, (1.f - cosTheta) * (1.f + cosTheta));
            u1 = phx_uniform(rng);
            u_maxSin2 = u1 * maxSin2;
            count += 1;
        } while (u_maxSin2 > sin2Theta && count < 100);
        if (count >= 100 && u_maxSin2 > sin2Theta) status |= PHX_STATUS_LOOP_CAP;
    }
    float sinTheta = sqrtf(sin2Theta);
    float u0 = phx_uniform(rng);
    float phi = 2.f * PHX_PI_F * u0;
    float sinPhi = sinf(phi);
    float cosPhi = cosf(phi);
    p.mom = make_float3(sinTheta * cosPhi, sinTheta * sinPhi, cosTheta);
    rotate_uz(p.mom, p0);
    p.pol = make_float3(cosTheta * cosPhi, cosTheta * sinPhi, -sinTheta);
    rotate_uz(p.pol, p0);
    p.wavelength = wavelength;
    float fraction, delta;
    {
        float NumberOfPhotons, N, u;
        float MeanMax = fmaxf(Mean1, Mean2);
        float DeltaN = (Mean1 - Mean2);
        unsigned count = 0;
        do {
            fraction = phx_uniform(rng);
            delta = fraction * step_length;
            NumberOfPhotons = Mean1 - fraction * DeltaN;
            u = phx_uniform(rng);
            N = u * MeanMax;
        } while (N > NumberOfPhotons && ++count < 100000);
        if (count >= 100000) status |= PHX_STATUS_LOOP_CAP;
    }
    float midVelocity = preVelocity + fraction * (postVelocity - preVelocity) * 0.5f;
    p.time = q1.w + delta / midVelocity;
    p.pos = make_float3(q1.x, q1.y, q1.z) + fraction * dpos;
    p.zero_flags();
    p.set_flag(PHX_CERENKOV);
}

// scarrier::generate sysrap/scarrier.h: the photon is the genstep's rows 2-5, moved 10 mm in y per photon
PHX_D void generate_carrier(PhxPhoton& p, const float4* g, unsigned long long photon_id)
{
    p.pos = make_float3(g[2].x, g[2].y + float(photon_id) * 10.f, g[2].z); p.time = g[2].w;
    p.mom = make_float3(g[3].x, g[3].y, g[3].z); p.hitcount_iindex = __float_as_uint(g[3].w);
    p.pol = make_float3(g[4].x, g[4].y, g[4].z); p.wavelength = g[4].w;
    p.obf = __float_as_uint(g[5].x); p.identity = __float_as_uint(g[5].y);
    p.index = __float_as_uint(g[5].z); p.flagmask = __float_as_uint(g[5].w);
    p.set_flag(PHX_TORCH);
}

// an sphoton (4 float4 rows) as given: an input photon (qudarap/qsim.h:2557, evt->photon[photon_id])
PHX_D void phx_load_sphoton(PhxPhoton& p, const float4* r)
{
    const float4 q0 = __ldg(r + 0), q1 = __ldg(r + 1), q2 = __ldg(r + 2), q3 = __ldg(r + 3);
    p.pos = make_float3(q0.x, q0.y, q0.z); p.time = q0.w;
    p.mom = make_float3(q1.x, q1.y, q1.z); p.hitcount_iindex = __float_as_uint(q1.w);
    p.pol = make_float3(q2.x, q2.y, q2.z); p.wavelength = q2.w;
    p.obf = __float_as_uint(q3.x); p.identity = __float_as_uint(q3.y);
    p.index = __float_as_uint(q3.z); p.flagmask = __float_as_uint(q3.w);
}

// qsim::generate_photon qudarap/qsim.h:2532-2561
// inlined into its callers: out of line, its photon and RNG state would go through local memory
PHX_D void generate_photon(PhxPhoton& p, curandStateXORWOW& rng, const float4* g, unsigned long long photon_id, const PhxProps& P, unsigned& status)
{
    const int gencode = __float_as_int(g[0].x);
    switch (gencode) {
        case PHX_GS_TORCH:
            generate_torch(p, rng, g, photon_id);
            if (p.wavelength <= 0.f) p.wavelength = tex2D<float>(P.planck_tex, curand_uniform(&rng), 0.5f);   // qplanck::wavelength
            break;
        case PHX_GS_G4Cerenkov_modified:
        case PHX_GS_CERENKOV: generate_cerenkov(p, rng, g, P, status); break;
        case PHX_GS_DsG4Scintillation_r4695:
        case PHX_GS_SCINTILLATION: generate_scint(p, rng, g, P); break;
        case PHX_GS_CARRIER: generate_carrier(p, g, photon_id); break;
        case PHX_GS_INPUT_PHOTON:
            if (P.input_photon && (long long)photon_id < P.num_input_photon) phx_load_sphoton(p, P.input_photon + 4 * photon_id);
            else status |= PHX_STATUS_INPUT_RANGE;
            p.set_flag(PHX_TORCH);
            break;
        default: break;
    }
    p.set_index(photon_id);
}

// ---------------------------------------------------------------- propagation
#define PHX_LOOP_CAP 1000000

PHX_COLD void rayleigh_scatter(PhxPhoton& p, curandStateXORWOW& rng, unsigned& status)
{
    float3 direction, polarization;
    bool looping = true;
    int count = 0;
    do {
        float u0 = phx_uniform(rng);
        float u1 = phx_uniform(rng);
        float u2 = phx_uniform(rng);
        float u3 = phx_uniform(rng);
        float u4 = phx_uniform(rng);
        float cosTheta = u0;
        float sinTheta = sqrtf(1.0f - u0 * u0);
        if (u1 < 0.5f) cosTheta = -cosTheta;
        float sinPhi, cosPhi;
        sincosf(2.f * PHX_PI_F * u2, &sinPhi, &cosPhi);
        direction = make_float3(sinTheta * cosPhi, sinTheta * sinPhi, cosTheta);
        rotate_uz(direction, p.mom);
        float constant = -dot(direction, p.pol);
        polarization.x = p.pol.x + constant * direction.x;
        polarization.y = p.pol.y + constant * direction.y;
        polarization.z = p.pol.z + constant * direction.z;
        if (dot(polarization, polarization) == 0.f) {
            sincosf(2.f * PHX_PI_F * u3, &sinPhi, &cosPhi);
            polarization = make_float3(cosPhi, sinPhi, 0.f);
            rotate_uz(polarization, direction);
        } else {
            if (u3 < 0.5f) polarization = -polarization;
        }
        polarization = normalize(polarization);
        float doCosTheta = dot(polarization, p.pol);
        float doCosTheta2 = doCosTheta * doCosTheta;
        looping = doCosTheta2 < u4;
    } while (looping && ++count < PHX_LOOP_CAP);
    if (looping) status |= PHX_STATUS_LOOP_CAP;
    p.mom = direction;
    p.pol = polarization;
}

// the pathwise tangent over one segment: the hit point's tangent and the change of the segment
// length (from the probe); on = the photon carries a nonzero tangent
struct PhxAdjSeg {
    bool on;
    float dD;
    float3 dpos_hit;
    float3 dnormal;
};

template <bool ADJ = false>
PHX_D int propagate_to_boundary(unsigned& flag, PhxPhoton& p, curandStateXORWOW& rng, const PhxState& s, float distance_to_boundary, const PhxProps& P, unsigned& status, PhxScore* sc = nullptr, const PhxAdjSeg* seg = nullptr)
{
    const bool scored = ADJ && s.m1idx == sc->mat;
    const bool carry = ADJ && seg && seg->on;
    const float absorption_length = s.material1.y;
    const float scattering_length = s.material1.z;
    const float reemission_prob = s.material1.w;
    const float group_velocity = s.m1group2.x;
    float u_scattering = phx_uniform(rng);
    float u_absorption = phx_uniform(rng);
    float scattering_distance = -scattering_length * logf(u_scattering);
    float absorption_distance = -absorption_length * logf(u_absorption);
    if (absorption_distance <= scattering_distance) {
        if (absorption_distance <= distance_to_boundary) {
            p.time += absorption_distance / group_velocity;
            p.pos += absorption_distance * (p.mom);
            float u_reemit = reemission_prob == 0.f ? 2.f : phx_uniform(rng);
            if (scored) {
                // absorbed at d (scattering later): log p = -log La - d/La - d/Ls ; then the reemission draw
                const float d = absorption_distance;
                score_add(*sc, 0, p.wavelength, -1.f / absorption_length + d / (absorption_length * absorption_length));
                score_add(*sc, 1, p.wavelength, d / (scattering_length * scattering_length));
                score_add(*sc, 2, p.wavelength, u_reemit < reemission_prob ? 1.f / reemission_prob : -1.f / (1.f - reemission_prob));
            }
            if (ADJ && carry) score_tangent_reset(*sc);   // a new wavelength and direction: nu changes
            if (u_reemit < reemission_prob) {
                float u_re_wavelength = phx_uniform(rng);
                float u_re_mom_ph = phx_uniform(rng);
                float u_re_mom_ct = phx_uniform(rng);
                float u_re_pol_ph = phx_uniform(rng);
                float u_re_pol_ct = phx_uniform(rng);
                p.wavelength = scint_wavelength(P, u_re_wavelength);
                p.mom = uniform_sphere(u_re_mom_ph, u_re_mom_ct);
                p.pol = normalize(cross(uniform_sphere(u_re_pol_ph, u_re_pol_ct), p.mom));
                flag = PHX_BULK_REEMIT;
                return PHX_CONTINUE;
            } else {
                flag = PHX_BULK_ABSORB;
                return PHX_BREAK;
            }
        }
    } else {
        if (scattering_distance <= distance_to_boundary) {
            if (scored) {
                const float d = scattering_distance;
                score_add(*sc, 1, p.wavelength, -1.f / scattering_length + d / (scattering_length * scattering_length));
                score_add(*sc, 0, p.wavelength, d / (absorption_length * absorption_length));
            }
            p.time += scattering_distance / group_velocity;
            p.pos += scattering_distance * (p.mom);
            const float3 e0 = p.pol;
            rayleigh_scatter(p, rng, status);
            if (ADJ && carry) {
                // the scattered direction d' is a path variable with density ~ 1 - (e.d')^2 about the
                // old polarisation e; the new polarisation is +-normalize(e - (e.d') d')
                const float3 d1 = p.mom, e1 = p.pol, de = sc->tpol;
                const float ed = dot(e0, d1);
                const float q = 1.f - ed * ed;
                if (q > 1e-12f) score_add_capped(*sc, p.wavelength, -2.f * ed * dot(de, d1) / q);
                const float3 u = e0 - ed * d1;
                const float ul = length(u);
                const float3 du = de - dot(de, d1) * d1;
                const float sgn = dot(e1, u) < 0.f ? -1.f : 1.f;
                sc->tpos = sc->tpos + scattering_distance * sc->tdir;
                sc->tdir = make_float3(0.f, 0.f, 0.f);
                sc->tpol = ul > 1e-12f ? (sgn / ul) * (du - dot(e1, du) * e1) : make_float3(0.f, 0.f, 0.f);
            }
            flag = PHX_BULK_SCATTER;
            return PHX_CONTINUE;
        }
    }
    if (scored) {
        // reached the boundary unabsorbed and unscattered: log p = -D/La - D/Ls
        const float D = distance_to_boundary;
        score_add(*sc, 0, p.wavelength, D / (absorption_length * absorption_length));
        score_add(*sc, 1, p.wavelength, D / (scattering_length * scattering_length));
    }
    if (ADJ && carry) {
        // the same survival with the segment length moved by the tangent, in whatever material
        score_add_capped(*sc, p.wavelength, -seg->dD * (1.f / absorption_length + 1.f / scattering_length));
        sc->tpos = seg->dpos_hit;
    }
    p.pos += distance_to_boundary * (p.mom);
    p.time += distance_to_boundary / group_velocity;
    return PHX_BOUNDARY;
}

#ifndef PHX_ADJ_TANGENT_CAP
#define PHX_ADJ_TANGENT_CAP 100.f
#endif
// d TransCoeff / d nu and the tangents of the new direction and polarisation: the arithmetic of
// propagate_at_boundary in dual numbers, with n1, n2, the direction, polarisation and surface
// normal carrying their derivatives; the branches (TIR, normal incidence, reflect) are the
// photon's own
PHX_D void adj_boundary_tangent(PhxScore& sc, const PhxPhoton& p, const PhxState& s, const float3& normal, const float3& dnormal,
                                bool tir, bool normal_incidence, bool reflect)
{
    const PhxDual one = dd(1.f, 0.f), two = dd(2.f, 0.f);
    const PhxDual n1 = dd(s.material1.x, s.m1idx == sc.mat ? 1.f : 0.f);
    const PhxDual n2 = dd(s.material2.x, s.m2idx == sc.mat ? 1.f : 0.f);
    const PhxDual eta = n1 / n2;
    const PhxDual3 mom = d3(p.mom, sc.tdir), pol = d3(p.pol, sc.tpol), nrm = d3(normal, dnormal);
    const PhxDual _c1 = -ddot(mom, nrm);
    const PhxDual3 on = _c1.v < 0.f ? d3(-1.f * nrm.v, -1.f * nrm.d) : nrm;
    const PhxDual3 trans = dcross(mom, on);
    const PhxDual trans_length = dsqrt(ddot(trans, trans));
    const PhxDual3 A_trans = normal_incidence ? pol : (one / trans_length) * trans;
    const PhxDual E1_perp = ddot(pol, A_trans);
    const PhxDual c1 = dfabs(_c1);
    const PhxDual c2 = tir ? dd(0.f, 0.f) : dsqrt(one - eta * eta * (one - c1 * c1));
    const PhxDual EdotN = ddot(pol, on);
    const PhxDual n1c1 = n1 * c1, n2c2 = n2 * c2, n2c1 = n2 * c1, n1c2 = n1 * c2;
    PhxDual E1x = dd(0.f, 0.f), E1y = dd(1.f, 0.f);
    if (!normal_incidence) {
        const PhxDual3 r = pol - E1_perp * A_trans;
        E1x = E1_perp;
        E1y = dsqrt(ddot(r, r));
    }
    const PhxDual tx = two * n1c1 * E1x / (n1c1 + n2c2);
    const PhxDual ty = two * n1c1 * E1y / (n2c1 + n1c2);
    const PhxDual T = (tir || n1c1.v == 0.f) ? dd(0.f, 0.f) : n2c2 * (tx * tx + ty * ty) / n1c1;
    if (!tir && T.v > 0.f && T.v < 1.f) {
        score_add_capped(sc, p.wavelength, (reflect ? -1.f / (1.f - T.v) : 1.f / T.v) * T.d);
    }
    const PhxDual3 mom2 = reflect ? mom + (two * c1) * on : eta * mom + (eta * c1 - c2) * on;
    PhxDual3 pol2;
    if (normal_incidence) {
        pol2 = reflect ? (s.material2.x > s.material1.x ? d3(-1.f * pol.v, -1.f * pol.d) : pol) : pol;
    } else if (reflect && tir) {
        pol2 = (two * EdotN) * on - pol;
    } else {
        const PhxDual3 A_paral = dnormalize(dcross(mom2, A_trans));
        const PhxDual rx = reflect ? tx - E1x : tx, ry = reflect ? (n2 * ty / n1) - E1y : ty;
        const PhxDual rl = dsqrt(rx * rx + ry * ry);
        pol2 = (rx / rl) * A_trans + (ry / rl) * A_paral;
    }
    // Near the critical angle the refracted direction's derivative grows without bound (d theta2/d n
    // ~ 1/cos theta2) while the transmission probability vanishes: the estimator's mean stays finite
    // but its variance does not.  The direction tangent is capped at PHX_ADJ_TANGENT_CAP (per unit
    // of n), a bias confined to rays refracted within about half a degree of grazing.
    const float tl = length(mom2.d), pl = length(pol2.d);
    sc.tdir = (tl > PHX_ADJ_TANGENT_CAP ? PHX_ADJ_TANGENT_CAP / tl : 1.f) * mom2.d;
    sc.tpol = (pl > PHX_ADJ_TANGENT_CAP ? PHX_ADJ_TANGENT_CAP / pl : 1.f) * pol2.d;
}

template <bool ADJ = false>
PHX_D int propagate_at_boundary(unsigned& flag, PhxPhoton& p, curandStateXORWOW& rng, const PhxState& s, const float3& normal, PhxScore* sc = nullptr, const PhxAdjSeg* seg = nullptr)
{
    const float n1 = s.material1.x;
    const float n2 = s.material2.x;
    const float eta = n1 / n2;
    const float _c1 = -dot(p.mom, normal);
    const float3 oriented_normal = _c1 < 0.f ? -normal : normal;
    const float3 trans = cross(p.mom, oriented_normal);
    const float trans_length = length(trans);
    const bool normal_incidence = trans_length < 1e-6f;
    const float3 A_trans = normal_incidence ? p.pol : trans / trans_length;
    const float E1_perp = dot(p.pol, A_trans);
    const float c1 = fabsf(_c1);
    const float c2c2 = 1.f - eta * eta * (1.f - c1 * c1);
    bool tir = c2c2 < 0.f;
    const float EdotN = dot(p.pol, oriented_normal);
    const float c2 = tir ? 0.f : sqrtf(c2c2);
    const float n1c1 = n1 * c1;
    const float n2c2 = n2 * c2;
    const float n2c1 = n2 * c1;
    const float n1c2 = n1 * c2;
    const float2 E1 = normal_incidence ? make_float2(0.f, 1.f) : make_float2(E1_perp, length(p.pol - (E1_perp * A_trans)));
    const float2 E2_t = make_float2(2.f * n1c1 * E1.x / (n1c1 + n2c2), 2.f * n1c1 * E1.y / (n2c1 + n1c2));
    const float2 E2_r = make_float2(E2_t.x - E1.x, (n2 * E2_t.y / n1) - E1.y);
    const float2 RR = normalize2(E2_r);
    const float2 TT = normalize2(E2_t);
    const float TransCoeff = (tir || n1c1 == 0.f ? 0.f : n2c2 * dot2(E2_t, E2_t) / n1c1);
    const float u_reflect = phx_uniform(rng);
    bool reflect = u_reflect > TransCoeff;
    if (ADJ && ((seg && seg->on) || s.m1idx == sc->mat || s.m2idx == sc->mat)) {
        // Fresnel branch probability log T (transmit) or log(1-T) (reflect) with T(n1, n2, incidence,
        // polarisation), and the new direction and polarisation tangents
        if (!(seg && seg->on)) score_tangent_reset(*sc);
        adj_boundary_tangent(*sc, p, s, normal, seg && seg->on ? seg->dnormal : make_float3(0.f, 0.f, 0.f), tir,
                             normal_incidence, reflect);
        if (!sc->pathwise) score_tangent_reset(*sc);
    }
    p.mom = reflect ? p.mom + 2.0f * c1 * oriented_normal : eta * (p.mom) + (eta * c1 - c2) * oriented_normal;
    const float3 A_paral = normalize(cross(p.mom, A_trans));
    p.pol = normal_incidence ? (reflect ? p.pol * (n2 > n1 ? -1.f : 1.f) : p.pol)
                             : (reflect ? (tir ? -p.pol + 2.f * EdotN * oriented_normal : RR.x * A_trans + RR.y * A_paral)
                                        : TT.x * A_trans + TT.y * A_paral);
    flag = reflect ? PHX_BOUNDARY_REFLECT : PHX_BOUNDARY_TRANSMIT;
    return PHX_CONTINUE;
}

PHX_D void random_direction_marsaglia(float3& dir, curandStateXORWOW& rng)
{
    float u0, u1, u, v, b, a;
    int count = 0;
    do {
        u0 = phx_uniform(rng);
        u1 = phx_uniform(rng);
        u = 2.f * u0 - 1.f;
        v = 2.f * u1 - 1.f;
        b = u * u + v * v;
    } while (b > 1.f && ++count < PHX_LOOP_CAP);
    a = 2.f * sqrtf(1.f - b);
    dir.x = a * u;
    dir.y = a * v;
    dir.z = 2.f * b - 1.f;
}

PHX_D void lambertian_direction(float3& dir, const float3& normal, float orient, curandStateXORWOW& rng)
{
    float ndotv;
    int count = 0;
    float u;
    do {
        count++;
        random_direction_marsaglia(dir, rng);
        ndotv = dot(dir, normal) * orient;
        if (ndotv < 0.f) {
            dir = -1.f * dir;
            ndotv = -1.f * ndotv;
        }
        u = phx_uniform(rng);
    } while (!(u < ndotv) && (count < 1024));
}

PHX_COLD void reflect_diffuse(PhxPhoton& p, curandStateXORWOW& rng, const float3& normal)
{
    float3 old_mom = p.mom;
    const float orient = dot(old_mom, normal) > 0.f ? -1.f : 1.f;
    lambertian_direction(p.mom, normal, orient, rng);
    float3 facet_normal = normalize(p.mom - old_mom);
    const float EdotN = dot(p.pol, facet_normal);
    p.pol = -1.f * (p.pol) + 2.f * EdotN * facet_normal;
}

PHX_D void reflect_specular(PhxPhoton& p, const float3& normal)
{
    const float PdotN = dot(p.mom, normal);
    p.mom = p.mom - 2.f * PdotN * normal;
    const float EdotN = dot(p.pol, normal);
    p.pol = -1.f * (p.pol) + 2.f * EdotN * normal;
}

PHX_D int propagate_at_surface(unsigned& flag, PhxPhoton& p, curandStateXORWOW& rng, const PhxState& s, const float3& normal)
{
    const float detect = s.surface.x;
    const float absorb = s.surface.y;
    const float reflect_diffuse_ = s.surface.w;
    float u_surface = phx_uniform(rng);
    int action = u_surface < absorb + detect ? PHX_BREAK : PHX_CONTINUE;
    if (action == PHX_BREAK) {
        flag = u_surface < absorb ? PHX_SURFACE_ABSORB : PHX_SURFACE_DETECT;
    } else {
        flag = u_surface < absorb + detect + reflect_diffuse_ ? PHX_SURFACE_DREFLECT : PHX_SURFACE_SREFLECT;
        if (flag == PHX_SURFACE_DREFLECT) reflect_diffuse(p, rng, normal);
        else reflect_specular(p, normal);
    }
    return action;
}

// The probe of the pathwise tangent: the prim the closest hit found, intersected along the ray moved
// by eps along the tangent (origin + eps tpos, direction + eps tdir); the differences give the
// hit point's tangent, the segment length's and the normal's.  A probe that misses the prim or
// lands on another face of it (normal turned by more than ~25 degrees) falls back to the
// tangent plane at the hit (no curvature).
#define PHX_ADJ_PROBE_SHIFT 10.f      // mm the probe moves the hit point
PHX_D void adj_probe(PhxAdjSeg& seg, const PhxScore& sc, const PhxPhoton& p, const PhxPRD& prd, unsigned& status)
{
    seg.on = sc.pathwise && !score_tangent_zero(sc);
    seg.dD = 0.f;
    seg.dpos_hit = make_float3(0.f, 0.f, 0.f);
    seg.dnormal = seg.dpos_hit;
    if (!seg.on) return;
    const float3 n1 = prd.normal;
    const float D = prd.distance;
    // tangent plane fallback: the hit point slides in the plane of the normal
    const float dn = dot(n1, p.mom);
    const float3 w = sc.tpos + D * sc.tdir;
    if (fabsf(dn) > 1e-6f) {
        seg.dD = -dot(n1, w) / dn;
        seg.dpos_hit = w + seg.dD * p.mom;
    }
    const float mag = length(sc.tpos) + D * length(sc.tdir);
    if (!(mag > 0.f) || !sc.prim_node) return;
    const float eps = PHX_ADJ_PROBE_SHIFT / mag;
    const float3 o2 = p.pos + eps * sc.tpos;
    const float3 d2 = normalize(p.mom + eps * sc.tdir);
    const unsigned gp = prd.gp_bd >> 16, ii = prd.ii_id >> 16;
    const float4* q = sc.inst_inv + 4 * ii;
    float4 m[4] = { __ldg(q + 0), __ldg(q + 1), __ldg(q + 2), __ldg(q + 3) };
    const float3 lo = xform_row(m, o2, 1.f), ld = xform_row(m, d2, 0.f);
    const float tmin = (p.obf & sc.eps0_mask) ? sc.tmin0 : sc.tmin;
    float4 is;
    unsigned st = 0;
    if (!intersect_prim<PHX_CV_FULL>(is, sc.csg, __ldg(sc.prim_node + gp), tmin, lo, ld, st)) return;
    const float3 n2 = normalize(xform_col(m, make_float3(is.x, is.y, is.z), 0.f));
    if (dot(n1, n2) < 0.9f) return;
    const float3 h1 = p.pos + D * p.mom;
    const float3 h2 = o2 + is.w * d2;
    seg.dD = (is.w - D) / eps;
    seg.dpos_hit = (1.f / eps) * (h2 - h1);
    seg.dnormal = (1.f / eps) * (n2 - n1);
    status |= st & PHX_STATUS_CSG_STACK;
}

// tangents through a surface: specular reflection as the mirror map (normal change included), a
// diffuse reflection draws a new direction (its density cos(angle to the normal) does not
// involve the old direction; the tangent restarts, the polarisation's change is not carried)
PHX_D void adj_surface_tangent(PhxScore& sc, unsigned flag, const float3& mom0, const float3& pol0, const float3& normal,
                               const float3& dnormal)
{
    if (flag == PHX_SURFACE_SREFLECT) {
        const PhxDual two = dd(2.f, 0.f);
        const PhxDual3 mom = d3(mom0, sc.tdir), pol = d3(pol0, sc.tpol), nrm = d3(normal, dnormal);
        const PhxDual3 mom2 = mom - (two * ddot(mom, nrm)) * nrm;
        const PhxDual3 pol2 = (two * ddot(pol, nrm)) * nrm - pol;
        sc.tdir = mom2.d;
        sc.tpol = pol2.d;
    } else if (flag == PHX_SURFACE_DREFLECT) {
        sc.tdir = make_float3(0.f, 0.f, 0.f);
        sc.tpol = sc.tdir;
    }
}

// qsim::propagate : returns CONTINUE/BREAK, sets the flag.  ADJ adds the score terms.
template <bool ADJ = false>
PHX_D int propagate(PhxPhoton& p, curandStateXORWOW& rng, const PhxPRD& prd, const PhxProps& P, unsigned& status, PhxScore* sc = nullptr)
{
    const unsigned boundary = prd.boundary();
    const unsigned identity = prd.identity();
    const unsigned iindex = prd.iindex();
    const float lposcost = prd.lposcost;
    const float3 normal = prd.normal;
    float cosTheta = dot(p.mom, normal);
    p.set_prd(boundary, identity, cosTheta, iindex);
    PhxState s;
    fill_state<ADJ>(s, P, boundary, p.wavelength, cosTheta);
    unsigned flag = 0;
    PhxAdjSeg seg;
    if (ADJ) adj_probe(seg, *sc, p, prd, status);
    int command = propagate_to_boundary<ADJ>(flag, p, rng, s, prd.distance, P, status, sc, ADJ ? &seg : nullptr);
    if (command == PHX_BOUNDARY) {
        const int ems = (int)s.optical.y;
        if (ems == PHX_EMS_NOSURFACE) {
            command = propagate_at_boundary<ADJ>(flag, p, rng, s, normal, sc, ADJ ? &seg : nullptr);
        } else if (ems == PHX_EMS_SURFACE || lposcost < 0.f) {
            float3 mom0 = p.mom, pol0 = p.pol;
            command = propagate_at_surface(flag, p, rng, s, normal);
            if (ADJ && seg.on) adj_surface_tangent(*sc, flag, mom0, pol0, normal, seg.dnormal);
        } else if (ems == PHX_EMS_SURFACE_ZPLUS_SENSOR_A) {
            (void)phx_uniform(rng);   // alignment burn of propagate_at_surface_Detect
            flag = PHX_SURFACE_DETECT;
            command = PHX_BREAK;
        }
    }
    p.set_flag(flag);
    return command;
}
