// esr_faithful.h -- launchers of the reference-fidelity float32 kernels.
//
// With esr_params.fidelity = ESR_FIDELITY_REFERENCE a float32 solver runs
// these instead of the fast float32 kernels: the same kernel templates with
// IEEE division, the reference's operation sequence and its per-call
// least-squares solve, compiled in esr_faithful.cu without FMA contraction so
// that every float32 operation rounds as the reference's float32 arithmetic
// does. Only that translation unit instantiates the float32 FAST = false
// kernels.
#pragma once
#include "esr_device.cuh"

namespace esr {

void faithful_recon(const BlockMap<float>& bm, const float4* W, float4* FV, long long total, const Cases<float>& cs,
                    const Consts<float>& kc, int pos, float* dt_local, bool muscl, bool localdt, int n_blk, int block,
                    cudaStream_t st);
// stage: ST_FIRST, ST_SRK2_SECOND or ST_RK2_SECOND
void faithful_flux(int stage, const BlockMap<float>& bm, const float4* win, const float4* wbase, float4* wout,
                   const float4* FV, long long total, const Cases<float>& cs, const Consts<float>& kc, int pos,
                   const float* dt_local, float* res, bool rusanov, bool muscl, bool localdt, int n_blk, int block,
                   cudaStream_t st);
// per-case minimum CFL step partials (k_case_reduce RED_DTMIN)
void faithful_dtmin(dim3 grid, int threads, const Seg<float>* segs, CaseMap cm, const float4* W, const int* due,
                    int chunk_cells, double2* partial, int n_chunks, const Consts<float>& kc, cudaStream_t st);

}  // namespace esr
