// esr_faithful.cu -- the reference-fidelity float32 kernels (built with
// -fmad=false: no multiply-add is fused, so each float32 product and sum
// rounds separately, as in the reference's float32 arithmetic).
#include "esr_faithful.h"

namespace esr {

void faithful_recon(const BlockMap<float>& bm, const float4* W, float4* FV, long long total, const Cases<float>& cs,
                    const Consts<float>& kc, int pos, float* dt_local, bool muscl, bool localdt, int n_blk, int block,
                    cudaStream_t st) {
  if (!muscl) {
    if (localdt) k_recon<float, false, false, true><<<n_blk, block, 0, st>>>(bm, W, nullptr, 0, cs, kc, pos, dt_local);
    return;
  }
  if (localdt) k_recon<float, false, true, true><<<n_blk, block, 0, st>>>(bm, W, FV, total, cs, kc, pos, dt_local);
  else k_recon<float, false, true, false><<<n_blk, block, 0, st>>>(bm, W, FV, total, cs, kc, pos, dt_local);
}

template <int STAGE>
static void flux_stage(const BlockMap<float>& bm, const float4* win, const float4* wbase, float4* wout,
                       const float4* FV, long long total, const Cases<float>& cs, const Consts<float>& kc, int pos,
                       const float* dt_local, float* res, bool rus, bool muscl, bool local, int n_blk, int block,
                       cudaStream_t st) {
#define ESR_FF(F, M, L)                                                                                      \
  if (rus == (F == 1) && muscl == M && local == L) {                                                         \
    k_flux<float, false, F, M, STAGE, L><<<n_blk, block, 0, st>>>(bm, win, wbase, wout, FV, total, cs, kc, pos, \
                                                                  dt_local, res);                            \
    return;                                                                                                  \
  }
  ESR_FF(0, true, false) ESR_FF(0, true, true) ESR_FF(0, false, false) ESR_FF(0, false, true)
  ESR_FF(1, true, false) ESR_FF(1, true, true) ESR_FF(1, false, false) ESR_FF(1, false, true)
#undef ESR_FF
}

void faithful_flux(int stage, const BlockMap<float>& bm, const float4* win, const float4* wbase, float4* wout,
                   const float4* FV, long long total, const Cases<float>& cs, const Consts<float>& kc, int pos,
                   const float* dt_local, float* res, bool rusanov, bool muscl, bool localdt, int n_blk, int block,
                   cudaStream_t st) {
  if (stage == ST_FIRST)
    flux_stage<ST_FIRST>(bm, win, wbase, wout, FV, total, cs, kc, pos, dt_local, res, rusanov, muscl, localdt, n_blk,
                         block, st);
  else if (stage == ST_SRK2_SECOND)
    flux_stage<ST_SRK2_SECOND>(bm, win, wbase, wout, FV, total, cs, kc, pos, dt_local, res, rusanov, muscl, localdt,
                               n_blk, block, st);
  else
    flux_stage<ST_RK2_SECOND>(bm, win, wbase, wout, FV, total, cs, kc, pos, dt_local, res, rusanov, muscl, localdt,
                              n_blk, block, st);
}

void faithful_dtmin(dim3 grid, int threads, const Seg<float>* segs, CaseMap cm, const float4* W, const int* due,
                    int chunk_cells, double2* partial, int n_chunks, const Consts<float>& kc, cudaStream_t st) {
  k_case_reduce<float, RED_DTMIN, false><<<grid, threads, 0, st>>>(segs, cm, W, nullptr, due, chunk_cells, partial,
                                                                   n_chunks, kc);
}

}  // namespace esr
