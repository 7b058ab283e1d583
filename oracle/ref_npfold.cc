// ref_npfold.cc : TEST INFRASTRUCTURE ONLY — writes geometry and material arrays with the
// reference's own array writer, so the loader is checked against files the reference would write.
//
// Compiled by oracle/Makefile (target `ref`) against the header-only sysrap/NP.hh where it lies in
// the reference checkout; the output goes to oracle/_ref/libref_npfold.so.  The two entry points
// mirror the reference's savers call for call:
//   ref_write_foundry  CSGFoundry::save_ (CSG/CSGFoundry.cc:2769-2800): NP::Write of solid (n,3,4)
//                      int32, prim/node/tran/itra/inst (n,4,4) float32, plan (n,1,4) float32,
//                      each only when it has rows; NP::WriteNames of meshname.txt
//   ref_write_standard sstandard (sysrap/sstandard.h:311-330, 495-506): bnd as NP::Make<double>
//                      (nb,4,2,nwl,4) with set_names and the domain_low/high/step/range metadata,
//                      optical as NP::Make<int> (nb,4,4); the scintillation icdf as a double array
//                      (QScint narrows it, qudarap/QScint.cc:41-44); saved with NP::save, which
//                      writes <name>_meta.txt and <name>_names.txt beside each .npy
#include <cstring>
#include <sstream>
#include <string>
#include <vector>
#include "NP.hh"

static std::vector<std::string> split_lines(const char* s)
{
    std::vector<std::string> out;
    if (!s) return out;
    std::stringstream ss(s);
    std::string line;
    while (std::getline(ss, line)) if (!line.empty()) out.push_back(line);
    return out;
}

extern "C" int ref_write_foundry(const char* dir, const int* solid, int ns, const float* prim, int np, const float* node, int nn,
                                 const float* tran, int nt, const float* itra, int nit, const float* inst, int ni,
                                 const float* plan, int npl, const char* meshnames)
{
    if (!dir) return -1;
    std::vector<std::string> meshname = split_lines(meshnames);
    if (meshname.size() > 0) NP::WriteNames(dir, "meshname.txt", meshname);
    if (ns > 0) NP::Write(dir, "solid.npy", solid, ns, 3, 4);
    if (np > 0) NP::Write(dir, "prim.npy", prim, np, 4, 4);
    if (nn > 0) NP::Write(dir, "node.npy", node, nn, 4, 4);
    if (npl > 0) NP::Write(dir, "plan.npy", plan, npl, 1, 4);
    if (nt > 0) NP::Write(dir, "tran.npy", tran, nt, 4, 4);
    if (nit > 0) NP::Write(dir, "itra.npy", itra, nit, 4, 4);
    if (ni > 0) NP::Write(dir, "inst.npy", inst, ni, 4, 4);
    return 0;
}

extern "C" int ref_write_standard(const char* dir, const double* bnd, int nb, int nwl, const char* bnd_names, const int* optical,
                                  const double* icdf, int icdf_ni, int icdf_nj, int icdf_nk, float domain_low, float domain_high,
                                  float domain_step)
{
    if (!dir || !bnd || !optical) return -1;
    NP* b = NP::Make<double>(nb, 4, 2, nwl, 4);
    memcpy(b->bytes(), bnd, b->arr_bytes());
    b->set_names(split_lines(bnd_names));
    b->set_meta<float>("domain_low", domain_low);
    b->set_meta<float>("domain_high", domain_high);
    b->set_meta<float>("domain_step", domain_step);
    b->set_meta<float>("domain_range", domain_high - domain_low);
    b->save(dir, "bnd.npy");
    NP* op = NP::Make<int>(nb, 4, 4);
    memcpy(op->bytes(), optical, op->arr_bytes());
    op->save(dir, "optical.npy");
    if (icdf && icdf_ni > 0) {
        NP* ic = NP::Make<double>(icdf_ni, icdf_nj, icdf_nk);
        memcpy(ic->bytes(), icdf, ic->arr_bytes());
        ic->save(dir, "icdf.npy");
        delete ic;
    }
    delete b;
    delete op;
    return 0;
}
