// ref_planck.cc : TEST INFRASTRUCTURE ONLY — the reference's black-body wavelength ICDF.
//
// Compiled by oracle/Makefile (target `ref`) with g++ against the unmodified reference header
// sysrap/sblackbody.h where it lies (with sysrap/NP.hh), into oracle/_ref/libref_planck.so.
// QPlanck builds the Planck texture from sblackbody<double>(4096, 4096, 6500 K, 80 nm, 800 nm)
// narrowed to float (qudarap/QPlanck.cc:36-48); this returns that table.
#include <cstring>
#include "sblackbody.h"

extern "C" int ref_planck_icdf(float* out, int n)
{
    sblackbody<double> bb(4096, 4096, 6500., 80., 800., 1000);
    const NP* icdf = bb.icdf;
    if (!icdf || icdf->num_values() != 4096 || n < 4096) return -1;
    const double* v = icdf->cvalues<double>();
    for (int i = 0; i < 4096; i++) out[i] = static_cast<float>(v[i]);
    return 0;
}
