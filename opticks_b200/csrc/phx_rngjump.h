// phx_rngjump.h : jump-ahead of XORWOW streams by whole events as one GF(2) matrix per event.
//
// The reference advances every photon's cuRAND XORWOW state by skipahead(event * 100000)
// (qudarap/qrng.h:85-90).  XORWOW is Marsaglia's xorshift recurrence on five 32-bit words plus a
// Weyl counter (G. Marsaglia, "Xorshift RNGs", J. Stat. Softw. 8(14), 2003):
//     t = x ^ (x >> 2); x = y; y = z; z = w; w = v; v = (v ^ (v << 4)) ^ (t ^ (t << 1)); d += 362437
// The five-word part is linear over GF(2), so n steps are one 160x160 bit matrix T^n, and the
// counter advances by 362437 n.  The host builds T from the recurrence, the powers
// P_k = T^(skip * 2^k) by repeated squaring, and the device composes M_e = prod_k P_k^(bit k of e)
// once per event (one thread per matrix column).  A photon then applies M_e to its 160-bit state:
// 160 predicated XORs of 32-byte columns instead of a multi-stage skipahead per photon, or, for a
// single event, 40 lookups in tables of M_e over 4-bit groups of the state (the "four Russians"
// grouping of a GF(2) matrix-vector product), built once per call.
// Matrices are stored column-major, one column = the image of one state bit, padded to 8 words.
#pragma once
#include <stdint.h>
#include <vector>

#include "phx_pod.h"                        // PHX_JUMP_BITS, PHX_JUMP_COLW, PHX_JUMP_MATW
#define PHX_JUMP_POWERS 32                       // events < 2^32

struct PhxV5 { uint32_t w[5]; };

// one step of the five-word recurrence (the Weyl counter is handled separately)
inline PhxV5 phx_xorwow_step(const PhxV5& s)
{
    const uint32_t t = s.w[0] ^ (s.w[0] >> 2);
    PhxV5 o;
    o.w[0] = s.w[1];
    o.w[1] = s.w[2];
    o.w[2] = s.w[3];
    o.w[3] = s.w[4];
    o.w[4] = (s.w[4] ^ (s.w[4] << 4)) ^ (t ^ (t << 1));
    return o;
}

// column-major 160x160 bit matrix, column c = image of state bit c
struct PhxJumpMat {
    std::vector<PhxV5> col;
    PhxJumpMat() : col(PHX_JUMP_BITS) {}
    static PhxJumpMat identity()
    {
        PhxJumpMat m;
        for (int c = 0; c < PHX_JUMP_BITS; c++) {
            for (int k = 0; k < 5; k++) m.col[c].w[k] = 0u;
            m.col[c].w[c >> 5] = 1u << (c & 31);
        }
        return m;
    }
    PhxV5 apply(const PhxV5& v) const
    {
        PhxV5 o = { { 0u, 0u, 0u, 0u, 0u } };
        for (int c = 0; c < PHX_JUMP_BITS; c++)
            if ((v.w[c >> 5] >> (c & 31)) & 1u)
                for (int k = 0; k < 5; k++) o.w[k] ^= col[c].w[k];
        return o;
    }
    // (this * b) : first b then this
    PhxJumpMat mul(const PhxJumpMat& b) const
    {
        PhxJumpMat r;
        for (int c = 0; c < PHX_JUMP_BITS; c++) r.col[c] = apply(b.col[c]);
        return r;
    }
};

inline PhxJumpMat phx_step_matrix()
{
    PhxJumpMat t;
    const PhxJumpMat id = PhxJumpMat::identity();
    for (int c = 0; c < PHX_JUMP_BITS; c++) t.col[c] = phx_xorwow_step(id.col[c]);
    return t;
}

inline PhxJumpMat phx_matrix_power(const PhxJumpMat& m, unsigned long long n)
{
    PhxJumpMat r = PhxJumpMat::identity(), b = m;
    while (n) {
        if (n & 1ull) r = b.mul(r);
        n >>= 1;
        if (n) b = b.mul(b);
    }
    return r;
}

// P_k = T^(skip * 2^k), k = 0..PHX_JUMP_POWERS-1, flattened for upload (column-major, padded)
inline std::vector<uint32_t> phx_jump_powers(unsigned long long skip)
{
    std::vector<uint32_t> out((size_t)PHX_JUMP_POWERS * PHX_JUMP_MATW, 0u);
    PhxJumpMat p = phx_matrix_power(phx_step_matrix(), skip);
    for (int k = 0; k < PHX_JUMP_POWERS; k++) {
        for (int c = 0; c < PHX_JUMP_BITS; c++)
            for (int w = 0; w < 5; w++) out[(size_t)k * PHX_JUMP_MATW + c * PHX_JUMP_COLW + w] = p.col[c].w[w];
        if (k + 1 < PHX_JUMP_POWERS) p = p.mul(p);
    }
    return out;
}
