// ref_spm.cu : TEST INFRASTRUCTURE ONLY — runs the reference's own hit merge on the GPU.
//
// Compiled by oracle/Makefile (target `ref`) with the reference's flags (--use_fast_math,
// sysrap/CMakeLists.txt:963) against sysrap/SPM.cu where it lies in the reference checkout;
// the output goes to oracle/_ref/libref_spm.so.  Host arrays in and out: the records are
// uploaded, SPM::merge_partial_select<sphoton|sphotonlite> runs on the default stream and the
// merged records come back.
#include <cstdio>
#include <cstring>
#include "SPM.cu"

template <typename T>
static int run(const void* h_in, long long n, unsigned mask, float tw, void* h_out, long long cap, long long* num_out)
{
    T* d_in = nullptr;
    if (cudaMalloc(&d_in, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess) return -2;
    if (n > 0) cudaMemcpy(d_in, h_in, sizeof(T) * n, cudaMemcpyHostToDevice);
    T* d_out = nullptr;
    size_t no = 0;
    SPM::merge_partial_select<T>(d_in, (size_t)n, &d_out, &no, mask, tw, 0);
    cudaError_t e = cudaDeviceSynchronize();
    *num_out = (long long)no;
    if (e == cudaSuccess && no > 0 && (long long)no <= cap) cudaMemcpy(h_out, d_out, sizeof(T) * no, cudaMemcpyDeviceToHost);
    if (d_out && d_out != d_in) cudaFree(d_out);
    cudaFree(d_in);
    e = cudaDeviceSynchronize();
    return e == cudaSuccess ? ((long long)no <= cap ? 0 : -3) : -2;
}

extern "C" int ref_spm_merge(const void* h_in, long long n, int lite, unsigned mask, float tw, void* h_out, long long cap,
                             long long* num_out)
{
    return lite ? run<sphotonlite>(h_in, n, mask, tw, h_out, cap, num_out)
                : run<sphoton>(h_in, n, mask, tw, h_out, cap, num_out);
}
