// esr_device.cuh -- device numerics and kernels of the explicit FVM solve.
//
// Every formula restates the EulerSR JAX solver (citations are paths inside
// the EulerSR checkout) with its evaluation order, so float32/float64 results
// track the reference's rounding; the data layout and the kernel split are
// this project's own:
//
//   state      W[item], item = seg.off + cell * B + slot  (one float4/double4
//              per cell and case, cases of one mesh innermost so a warp of a
//              batched mesh walks 32 cases of the same cell: every geometry
//              load is a broadcast and every branch on boundary type uniform)
//   geometry   per mesh, one record of G_COUNT values per cell
//              (geo[cell * G_COUNT + field], esr_layout.h), read as float4/double4 groups
//   K1 recon   cell + 3 neighbour primitives, LSQ gradient, Venkatakrishnan
//              limiter, the 3 MUSCL face states of the cell -> FV[k][item]
//   K2 flux    per cell: the 3 face fluxes (HLLC or Rusanov) from its own
//              face states and its neighbours' face states on the shared
//              faces, sum / area, sponge, Runge-Kutta stage update. Each cell
//              owns its residual (no atomics); the sum order is fixed.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "esr_layout.h"

namespace esr {

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };
template <typename T> using V4 = typename Vec4<T>::type;

template <typename T> __host__ __device__ inline V4<T> mk4(T a, T b, T c, T d) {
  V4<T> r; r.x = a; r.y = b; r.z = c; r.w = d; return r;
}

template <typename T>
struct Seg {                 // one mesh and its B case slots
  int n_cells;
  int B;                     // case slots on this mesh
  int case0;                 // global slot index of slot 0
  int geo_stride;            // G_COUNT (values per cell record)
  long long off;             // first item of this segment in the state arrays
  const int4* nbr;           // x,y,z neighbour cell (-1 boundary), w packed slot info
  const T* geo;              // per-cell records of G_COUNT values
  const int* wall_cell;      // force faces: owner cell
  const T* wall_nx;          // owner's outward unit normal
  const T* wall_ny;
  const T* wall_ds;          // face length
  const LsqRef* lsq;         // per-cell least-squares data (reference-fidelity float32 only)
  const int* patch_start;    // first cell of every patch of the renumbering (+ n_cells)
  const int4* live;          // (A, magic, shift, -): slots 0..A-1 may hold running cases (A = B
                             // until a batch's queue is empty and its running cases are packed)
  int n_patches;
  int n_wall;
  int b_shift;               // item / B = (umulhi(item, b_magic) + item) >> b_shift
  unsigned b_magic;
  int pad;
};

// cell of an item of segment s without an integer divide (items < 2^31;
// multiplier and shift chosen on the host, checked there against n / B)
template <typename T>
__device__ __forceinline__ int cell_of(const Seg<T>& s, int item) {
  return (int)((__umulhi((unsigned)item, s.b_magic) + (unsigned)item) >> s.b_shift);
}

// cell and slot of thread item `item` of segment s: items walk (cell, slot)
// over the first A slots of every cell, A = live slots (B until a batch's
// queue drains and compaction packs its running cases into slots 0..A-1),
// so once few cases remain the work lands on few warps with full lanes. A
// one-slot segment has no live record (s.live null: nothing to pack), which
// spares its small, latency-bound launches the dependent load.
template <typename T>
__device__ __forceinline__ bool item_slot(const Seg<T>& s, int item, int& c, int& b) {
  int4 L = make_int4(s.B, 0, 0, 0);
  if (s.live != nullptr) L = *s.live;
  if (L.x == s.B) {
    if (item >= s.n_cells * s.B) return false;
    c = cell_of(s, item);
    b = item - c * s.B;
  } else {
    if (item >= s.n_cells * L.x) return false;
    c = (int)divide((unsigned)item, Divider{(unsigned)L.y, L.z});
    b = item - c * L.x;
  }
  return true;
}

// Which segment and first item a block of the cell kernels covers. A
// one-mesh solver passes its segment by value (kernel parameters live in the
// constant bank) so the block needs no table lookups; several meshes go
// through the block table (mesh segment, first item).
template <typename T>
struct BlockMap {
  const Seg<T>* segs;
  const int2* blk;
  Seg<T> seg0;
  int single;
};

template <typename T>
__device__ __forceinline__ void block_origin(const BlockMap<T>& bm, Seg<T>& s, int& first) {
  if (bm.single) {
    s = bm.seg0;
    first = blockIdx.x * blockDim.x;
  } else {
    const int2 bt = bm.blk[blockIdx.x];
    s = bm.segs[bt.x];
    first = bt.y;
  }
}

// Precision policy. FAST = false keeps IEEE division and the reference's
// exact operation sequence: every float64 kernel, and the float32 kernels of
// the reference-fidelity mode (compiled without FMA contraction in their own
// translation unit, esr_faithful.cu). FAST float32 kernels (the default) use
// the approximate divide (div.approx, <= 2 ulp) and reciprocal-multiplies.
template <typename T, bool FAST> constexpr bool kFastPath = FAST && sizeof(T) == 4;
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ T dv(T a, T b) {
  if constexpr (kFastPath<T, FAST>) return __fdividef(a, b);
  else return a / b;
}

// Resident 256-thread blocks per SM the float32 cell kernels are compiled for
// (register caps 65536 / (256 x n)); float64 kernels take what they need.
#ifndef ESR_K1_MINB
#define ESR_K1_MINB 8
#endif
#ifndef ESR_K1_MINB_LOCAL
#define ESR_K1_MINB_LOCAL 4
#endif
#ifndef ESR_K2_MINB
#define ESR_K2_MINB 5   // 48 registers: 7-9 % faster than 4 blocks (62 registers), no spills
#endif
// The autotuner's second register budget of each fast float32 kernel; a
// kernel's MINB template argument of 0 means the default above.
#ifndef ESR_K1_MINB_ALT
#define ESR_K1_MINB_ALT 6
#endif
#ifndef ESR_K2_MINB_ALT
#define ESR_K2_MINB_ALT 4
#endif
template <typename T, bool FAST, int MINB, int DEF>
constexpr int kMinBlocks = kFastPath<T, FAST> ? (MINB ? MINB : DEF) : 1;

template <typename T>
struct Consts {
  T gamma, gm1;              // run gamma and gamma - 1 rounded from double
  T inv_gm1, inv_gm1_14;     // 1/(gamma-1), 1/(1.4-1) for the float32 path
  T gm1_14;                  // 1.4 - 1 (wall ghost and forces use gamma 1.4)
  T half, eps_lim, venk_eps; // 0.5, limiter threshold, Venkatakrishnan 1e-7
  T ss_eps, den_eps;         // HLLC 1e-6 wave-speed split, 1e-12 denominator guard
  T sub_rho, sub_u, sub_v;   // subsonic inlet primitives
};

template <typename T>
struct Cases {               // per global slot
  const T* dt;
  const V4<T>* inlet;        // conserved inlet state
  const T* strength;         // sponge strength (|U_inf| + a_inf) / width
  const int* active;
  const int* step;           // steps done at the start of the current chunk
  const int* nmax;
};

// ----------------------------------------------------------- conversions
// helper.py:37-46 getPrimitive (M = 1)
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ void prim(const V4<T>& W, T gm1, T half, T P[4]) {
  T r = W.x;
  T u, v;
  if constexpr (kFastPath<T, FAST>) {
    const T ri = __fdividef(1.0f, r);
    u = W.y * ri;
    v = W.z * ri;
  } else {
    u = W.y / r;
    v = W.z / r;
  }
  P[0] = r; P[1] = u; P[2] = v;
  P[3] = (W.w - half * r * (u * u + v * v)) * gm1;
}
// helper.py:25-35 getConserved (M = 1)
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ V4<T> cons(const T P[4], T gm1, T inv_gm1, T half) {
  T r = P[0], u = P[1], v = P[2];
  const T e = kFastPath<T, FAST> ? P[3] * inv_gm1 : P[3] / gm1;
  return mk4<T>(r, r * u, r * v, e + half * r * (u * u + v * v));
}

// helper.py:196-204 slip wall ghost (gamma 1.4, background value 0)
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ V4<T> wall_ghost(const V4<T>& Wc, T nx, T ny, const Consts<T>& k) {
  T P[4];
  prim<T, FAST>(Wc, k.gm1_14, k.half, P);
  T vn = P[1] * nx + P[2] * ny;
  T Q[4] = {P[0], P[1] - T(2) * vn * nx, P[2] - T(2) * vn * ny, P[3]};
  return cons<T, FAST>(Q, k.gm1_14, k.inv_gm1_14, k.half);
}
// helper.py:179-194 subsonic inlet ghost: rho,u,v imposed, p from the cell (gamma 1.4)
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ V4<T> subsonic_ghost(const V4<T>& Wc, const Consts<T>& k) {
  T P[4];
  prim<T, FAST>(Wc, k.gm1_14, k.half, P);
  T Q[4] = {k.sub_rho, k.sub_u, k.sub_v, P[3]};
  return cons<T, FAST>(Q, k.gm1_14, k.inv_gm1_14, k.half);
}
// helper.py:233-256 BC_state for one boundary slot (conserved ghost)
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ V4<T> ghost_cons(int kind, const V4<T>& Wc, T nx, T ny, const V4<T>& inlet,
                                            const Consts<T>& k) {
  if (kind == K_WALL) return wall_ghost<T, FAST>(Wc, nx, ny, k);
  if (kind == K_INLET) return inlet;
  if (kind == K_SUBSONIC) return subsonic_ghost<T, FAST>(Wc, k);
  return Wc;  // outlet
}

// euler_solver.py:36-39 Venkatakrishnan with K = 0
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ T venkat(T a, T b, T eps) {
  return dv<T, FAST>(a * a + T(2) * a * b, a * a + T(2) * b * b + a * b + eps);
}

// ------------------------------------------------------------------ fluxes
// euler_solver.py:376-420 getFlux with the HLLC dissipation of :273-374;
// returns Fc - (Fc - F_HLLC) exactly as the reference assembles it.
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ void hllc(const V4<T>& WL, const T PL[4], const V4<T>& WR, const T PR[4],
                                     T nx, T ny, const Consts<T>& k, T F[4]) {
  const T rL = PL[0], uL = PL[1], vL = PL[2], pL = PL[3];
  const T rR = PR[0], uR = PR[1], vR = PR[2], pR = PR[3];
  const T unL = uL * nx + vL * ny;
  const T unR = uR * nx + vR * ny;
  const T tx = -ny, ty = nx;
  const T utL = uL * tx + vL * ty;
  const T utR = uR * tx + vR * ty;
  const T aL = sqrt(fabs(dv<T, FAST>(k.gamma * pL, rL)));
  const T aR = sqrt(fabs(dv<T, FAST>(k.gamma * pR, rR)));
  T SL = fmin(unL - aL, unR - aR);
  T SR = fmax(unL + aL, unR + aR);
  if (SL == SR) SL = SL - k.ss_eps;
  if (SL == SR) SR = SR + k.ss_eps;
  const T EL = WL.w, ER = WR.w;
  T den = rL * (SL - unL) - rR * (SR - unR);
  if (den == T(0)) den = k.den_eps;
  const T Ss = dv<T, FAST>(pR - pL + rL * unL * (SL - unL) - rR * unR * (SR - unR), den);
  const T PsL = pL + rL * (SL - unL) * (Ss - unL);
  const T PsR = pR + rR * (SR - unR) * (Ss - unR);
  const T Ps = k.half * (PsL + PsR);
  // jnp.where cascade of :369-371; the star state is built once for the side it needs
  const bool c1 = SL >= T(0);
  const bool c2 = (SL <= T(0)) && (Ss >= T(0));
  const bool c3 = (Ss <= T(0)) && (SR >= T(0));
  const bool left = c1 || c2;
  const T rK = left ? rL : rR, unK = left ? unL : unR, SK = left ? SL : SR;
  const T EK = left ? EL : ER, pK = left ? pL : pR, utK = left ? utL : utR;
  if constexpr (kFastPath<T, FAST>) {
    // float32: the HLLC flux itself (the central-flux identity F = Fc - (Fc - H)
    // is exact in real arithmetic) and only the physical flux of the selected side
    const T uK = left ? uL : uR, vK = left ? vL : vR;
    const V4<T> WK = left ? WL : WR;
    const T FK0 = rK * unK, FK1 = rK * uK * unK + pK * nx, FK2 = rK * vK * unK + pK * ny, FK3 = (EK + pK) * unK;
    if (left ? !c1 : c3) {
      const T inv = __fdividef(1.0f, SK - Ss);
      const T rs = rK * (SK - unK) * inv;
      const T Us3 = ((SK - unK) * EK - pK * unK + Ps * Ss) * inv;
      const T Us1 = rs * (Ss * nx + utK * tx), Us2 = rs * (Ss * ny + utK * ty);
      F[0] = FK0 + SK * (rs - WK.x);
      F[1] = FK1 + SK * (Us1 - WK.y);
      F[2] = FK2 + SK * (Us2 - WK.z);
      F[3] = FK3 + SK * (Us3 - WK.w);
    } else {
      F[0] = FK0; F[1] = FK1; F[2] = FK2; F[3] = FK3;
    }
  } else {
    const T FL0 = rL * unL, FL1 = rL * uL * unL + pL * nx, FL2 = rL * vL * unL + pL * ny, FL3 = (EL + pL) * unL;
    const T FR0 = rR * unR, FR1 = rR * uR * unR + pR * nx, FR2 = rR * vR * unR + pR * ny, FR3 = (ER + pR) * unR;
    const T Fc0 = k.half * (FL0 + FR0), Fc1 = k.half * (FL1 + FR1);
    const T Fc2 = k.half * (FL2 + FR2), Fc3 = k.half * (FL3 + FR3);
    const T rs = rK * (SK - unK) / (SK - Ss);
    const T Us3 = ((SK - unK) * EK - pK * unK + Ps * Ss) / (SK - Ss);
    const T Us0 = rs, Us1 = rs * (Ss * nx + utK * tx), Us2 = rs * (Ss * ny + utK * ty);
    T H0, H1, H2, H3;
    if (c1) { H0 = FL0; H1 = FL1; H2 = FL2; H3 = FL3; }
    else if (c2) { H0 = FL0 + SL * (Us0 - WL.x); H1 = FL1 + SL * (Us1 - WL.y); H2 = FL2 + SL * (Us2 - WL.z); H3 = FL3 + SL * (Us3 - WL.w); }
    else if (c3) { H0 = FR0 + SR * (Us0 - WR.x); H1 = FR1 + SR * (Us1 - WR.y); H2 = FR2 + SR * (Us2 - WR.z); H3 = FR3 + SR * (Us3 - WR.w); }
    else { H0 = FR0; H1 = FR1; H2 = FR2; H3 = FR3; }
    F[0] = Fc0 - (Fc0 - H0); F[1] = Fc1 - (Fc1 - H1);
    F[2] = Fc2 - (Fc2 - H2); F[3] = Fc3 - (Fc3 - H3);
  }
}

// euler_solver.py:203-240 Rusanov (plain branch) inside getFlux
template <typename T, bool FAST = (sizeof(T) == 4)>
__device__ __forceinline__ void rusanov(const V4<T>& WL, const T PL[4], const V4<T>& WR, const T PR[4],
                                        T nx, T ny, const Consts<T>& k, T F[4]) {
  const T unL = PL[1] * nx + PL[2] * ny;
  const T unR = PR[1] * nx + PR[2] * ny;
  const T FL0 = PL[0] * unL, FL1 = PL[0] * PL[1] * unL + PL[3] * nx, FL2 = PL[0] * PL[2] * unL + PL[3] * ny, FL3 = (WL.w + PL[3]) * unL;
  const T FR0 = PR[0] * unR, FR1 = PR[0] * PR[1] * unR + PR[3] * nx, FR2 = PR[0] * PR[2] * unR + PR[3] * ny, FR3 = (WR.w + PR[3]) * unR;
  const T CL = sqrt(fabs(dv<T, FAST>(k.gamma * PL[3], PL[0]))) + fabs(unL);
  const T CR = sqrt(fabs(dv<T, FAST>(k.gamma * PR[3], PR[0]))) + fabs(unR);
  const T C = fmax(CR, CL);
  F[0] = k.half * (FL0 + FR0) - k.half * C * (WR.x - WL.x);
  F[1] = k.half * (FL1 + FR1) - k.half * C * (WR.y - WL.y);
  F[2] = k.half * (FL2 + FR2) - k.half * C * (WR.z - WL.z);
  F[3] = k.half * (FL3 + FR3) - k.half * C * (WR.w - WL.w);
}

template <typename T>
__device__ __forceinline__ T geo(const Seg<T>& s, int f, int c) { return __ldg(s.geo + (size_t)c * G_COUNT + f); }

// N4 consecutive groups of 4 geometry values of cell c, from group g0, as
// vector loads (the per-cell record is 16-byte aligned)
template <typename T, int N4>
__device__ __forceinline__ void geo_groups(const Seg<T>& s, int c, int g0, T out[4 * N4]) {
  const V4<T>* p = reinterpret_cast<const V4<T>*>(s.geo + (size_t)c * G_COUNT) + g0;
#pragma unroll
  for (int i = 0; i < N4; ++i) {
    const V4<T> v = p[i];
    out[4 * i] = v.x; out[4 * i + 1] = v.y; out[4 * i + 2] = v.z; out[4 * i + 3] = v.w;
  }
}

// --------------------------------------------------------------- K1 recon
// euler_solver.py:106-122 build_reconstruction for MUSCL: BC ghosts, LSQ
// gradient (helper.py:136-153), limiter (euler_solver.py:45-67) and the cell's
// own MUSCL face states (euler_solver.py:69-98). Writes FV[k][item] (primitive).
// With LOCALDT it also writes the per-cell CFL time step of the state.
// MUSCL=false only computes the local dt (constant reconstruction needs no face states).
template <typename T, bool FAST, bool MUSCL, bool LOCALDT, int MINB = 0>
__global__ void __launch_bounds__(256, (kMinBlocks<T, FAST, MINB, LOCALDT ? ESR_K1_MINB_LOCAL : ESR_K1_MINB>)) k_recon(const BlockMap<T> bm,
                                               const V4<T>* __restrict__ W, V4<T>* __restrict__ FV,
                                               long long total, Cases<T> cs, Consts<T> kc, int pos,
                                               T* __restrict__ dt_local) {
  Seg<T> s;
  int first;
  block_origin(bm, s, first);
  int c, b;
  if (!item_slot(s, first + threadIdx.x, c, b)) return;
  const int g = s.case0 + b;
  if (!cs.active[g] || cs.step[g] + pos >= cs.nmax[g]) return;
  const long long gi = s.off + (long long)c * s.B + b;
  const V4<T> Wc = W[gi];
  T Pc[4];
  prim<T, FAST>(Wc, kc.gm1, kc.half, Pc);
  if (LOCALDT) {
    T gn[12];
    geo_groups<T, 3>(s, c, 0, gn);
    const T cel = sqrt(fabs(kc.gamma * Pc[3] / Pc[0]));
    T lam = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T un = Pc[1] * gn[G_N0X + 2 * k] + Pc[2] * gn[G_N0Y + 2 * k];
      const T term = (cel + fabs(un)) * gn[G_S0 + k];
      lam = (k == 0) ? term : lam + term;
    }
    dt_local[gi] = gn[G_AREA] / lam * cs.dt[g];   // cs.dt holds the case CFL in local mode
  }
  if (!MUSCL) return;
  const int4 nb = __ldg(s.nbr + c);
  const int nbk[3] = {nb.x, nb.y, nb.z};
  T Pk[3][4];
  const V4<T> inlet = cs.inlet[g];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int kind = slot_kind(nb.w, k);
    V4<T> Wk;
    if (kind == K_INTERIOR) Wk = W[s.off + (long long)nbk[k] * s.B + b];
    else Wk = ghost_cons<T, FAST>(kind, Wc, geo(s, G_N0X + 2 * k, c), geo(s, G_N0Y + 2 * k, c), inlet, kc);
    prim<T, FAST>(Wk, kc.gm1, kc.half, Pk[k]);
  }
  T gc[12];   // LSQ coefficients and face offsets (groups 3-5)
  geo_groups<T, 3>(s, c, 3, gc);
  T gx[4], gy[4];
  if constexpr (!FAST && sizeof(T) == 4) {
    // helper.py:136-153 per call, in the reference's float32 rounding:
    // b = sum_k (w_k dW_k) dx_k summed k = 0, 1, 2 in turn, then the 2x2
    // solve with partial pivoting in float64 rounded to float32 (what
    // numpy.linalg.solve computes for float32 operands)
    const LsqRef L = s.lsq[c];
    const double a00 = L.a[0], a01 = L.a[1], a10 = L.a[2], a11 = L.a[3];
    const bool sw = fabs(a10) > fabs(a00);
    const double p00 = sw ? a10 : a00, p01 = sw ? a11 : a01, p10 = sw ? a00 : a10, p11 = sw ? a01 : a11;
    const double l = p10 * (1.0 / p00), u11 = p11 - l * p01;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const T d0 = Pk[0][v] - Pc[v], d1 = Pk[1][v] - Pc[v], d2 = Pk[2][v] - Pc[v];
      const T x0 = L.w[0] * d0, x1 = L.w[1] * d1, x2 = L.w[2] * d2;
      const T bx = (x0 * L.dx[0] + x1 * L.dx[2]) + x2 * L.dx[4];
      const T by = (x0 * L.dx[1] + x1 * L.dx[3]) + x2 * L.dx[5];
      const double q0 = sw ? by : bx, q1 = sw ? bx : by;
      const double s1 = (q1 - l * q0) / u11;
      const double s0 = (q0 - p01 * s1) / p00;
      gx[v] = (T)s0;
      gy[v] = (T)s1;
    }
  } else {
    const T c0x = gc[G_C0X - 12], c0y = gc[G_C0Y - 12], c1x = gc[G_C1X - 12], c1y = gc[G_C1Y - 12];
    const T c2x = gc[G_C2X - 12], c2y = gc[G_C2Y - 12];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const T d0 = Pk[0][v] - Pc[v], d1 = Pk[1][v] - Pc[v], d2 = Pk[2][v] - Pc[v];
      gx[v] = c0x * d0 + c1x * d1 + c2x * d2;
      gy[v] = c0y * d0 + c1y * d1 + c2y * d2;
    }
  }
  const T fx[3] = {gc[G_F0X - 12], gc[G_F1X - 12], gc[G_F2X - 12]};
  const T fy[3] = {gc[G_F0Y - 12], gc[G_F1Y - 12], gc[G_F2Y - 12]};
  T phi[4], D[3][4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const T mn = fmin(fmin(Pc[v], Pk[0][v]), fmin(Pk[1][v], Pk[2][v]));
    const T mx = fmax(fmax(Pc[v], Pk[0][v]), fmax(Pk[1][v], Pk[2][v]));
    // min over the three faces only: the Venkatakrishnan value can exceed 1
    T ph = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T d = fx[k] * gx[v] + fy[k] * gy[v];
      D[k][v] = d;
      T p = T(1);
      if (d > kc.eps_lim) p = venkat<T, FAST>(mx - Pc[v], d, kc.venk_eps);
      else if (d < -kc.eps_lim) p = venkat<T, FAST>(mn - Pc[v], d, kc.venk_eps);
      ph = (k == 0) ? p : fmin(ph, p);
    }
    phi[v] = ph;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int kind = slot_kind(nb.w, k);
    V4<T> o;
    if (kind == K_INTERIOR)
      o = mk4<T>(Pc[0] + phi[0] * D[k][0], Pc[1] + phi[1] * D[k][1], Pc[2] + phi[2] * D[k][2], Pc[3] + phi[3] * D[k][3]);
    else
      o = mk4<T>(Pc[0], Pc[1], Pc[2], Pc[3]);
    FV[(long long)k * total + gi] = o;
  }
}

// Unlimited LSQ gradient of the primitives with boundary ghosts, as the
// bundle export computes it (euler/utils.py:33-39 -> helper.py:136-153), for
// one slot; out[(c*4 + v)*2 + d] in the caller's cell order.
template <typename T>
__global__ void k_grad_export(const Seg<T>* __restrict__ segs, int seg, int b, const V4<T>* __restrict__ W,
                              const V4<T>* __restrict__ inlet_p, const int* __restrict__ inv, int g_slot,
                              Consts<T> kc, double* __restrict__ out) {
  const Seg<T> s = segs[seg];
  const int cc = blockIdx.x * blockDim.x + threadIdx.x;   // caller order
  if (cc >= s.n_cells) return;
  const int c = inv[cc];
  const long long gi = s.off + (long long)c * s.B + b;
  const V4<T> Wc = W[gi];
  T Pc[4];
  prim<T>(Wc, kc.gm1, kc.half, Pc);
  const int4 nb = __ldg(s.nbr + c);
  const int nbk[3] = {nb.x, nb.y, nb.z};
  const V4<T> inlet = inlet_p[g_slot];
  T Pk[3][4];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int kind = slot_kind(nb.w, k);
    V4<T> Wk;
    if (kind == K_INTERIOR) Wk = W[s.off + (long long)nbk[k] * s.B + b];
    else Wk = ghost_cons<T>(kind, Wc, geo(s, G_N0X + 2 * k, c), geo(s, G_N0Y + 2 * k, c), inlet, kc);
    prim<T>(Wk, kc.gm1, kc.half, Pk[k]);
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const T d0 = Pk[0][v] - Pc[v], d1 = Pk[1][v] - Pc[v], d2 = Pk[2][v] - Pc[v];
    out[((size_t)cc * 4 + v) * 2 + 0] = (double)(geo(s, G_C0X, c) * d0 + geo(s, G_C1X, c) * d1 + geo(s, G_C2X, c) * d2);
    out[((size_t)cc * 4 + v) * 2 + 1] = (double)(geo(s, G_C0Y, c) * d0 + geo(s, G_C1Y, c) * d1 + geo(s, G_C2Y, c) * d2);
  }
}

// ----------------------------------------------------------------- K2 flux
enum Stage { ST_FIRST = 0, ST_SRK2_SECOND = 1, ST_RK2_SECOND = 2 };

// ---- the fast float32 face flux and cell update with every rounding written
// out (__fmul_rn / __fadd_rn / __fsub_rn / __fmaf_rn are never fused or
// split by the compiler), so the per-cell K2 and K2 by patches, which reach
// the same faces from different code, round every face flux and every cell
// update identically: a case's result does not depend on which K2 ran.
namespace xr {
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// helper.py:37-46 (M = 1)
__device__ __forceinline__ void prim(const float4& W, float gm1, float half, float P[4]) {
  const float r = W.x, ri = __fdividef(1.0f, r);
  const float u = mul(W.y, ri), v = mul(W.z, ri);
  P[0] = r; P[1] = u; P[2] = v;
  P[3] = mul(sub(W.w, mul(mul(half, r), fma(u, u, mul(v, v)))), gm1);
}
// helper.py:25-35 (M = 1)
__device__ __forceinline__ float4 cons(const float P[4], float inv_gm1, float half) {
  const float r = P[0], u = P[1], v = P[2];
  return make_float4(r, mul(r, u), mul(r, v), fma(mul(half, r), fma(u, u, mul(v, v)), mul(P[3], inv_gm1)));
}
// helper.py:233-256 boundary states, as primitives of the ghost (gamma 1.4)
__device__ __forceinline__ void ghost_prim(int kind, const float4& Wc, float nx, float ny, const float4& inlet,
                                           const Consts<float>& k, float Q[4]) {
  float P[4];
  if (kind == K_INLET) { prim(inlet, k.gm1, k.half, Q); return; }
  if (kind != K_WALL && kind != K_SUBSONIC) { prim(Wc, k.gm1, k.half, Q); return; }   // outlet
  prim(Wc, k.gm1_14, k.half, P);
  float G[4];
  if (kind == K_WALL) {       // helper.py:196-204
    const float t = mul(2.0f, fma(P[1], nx, mul(P[2], ny)));
    G[0] = P[0]; G[1] = sub(P[1], mul(t, nx)); G[2] = sub(P[2], mul(t, ny)); G[3] = P[3];
  } else {                    // helper.py:179-194
    G[0] = k.sub_rho; G[1] = k.sub_u; G[2] = k.sub_v; G[3] = P[3];
  }
  prim(cons(G, k.inv_gm1_14, k.half), k.gm1, k.half, Q);
}
// euler_solver.py:273-374 HLLC flux from the face primitives, the conserved
// variables formed only for the side the wave fan selects
__device__ __forceinline__ void hllc(const float PL[4], const float PR[4], float nx, float ny,
                                     const Consts<float>& k, float F[4]) {
  const float rL = PL[0], uL = PL[1], vL = PL[2], pL = PL[3];
  const float rR = PR[0], uR = PR[1], vR = PR[2], pR = PR[3];
  const float unL = fma(uL, nx, mul(vL, ny)), unR = fma(uR, nx, mul(vR, ny));
  const float tx = -ny, ty = nx;
  const float aL = sqrtf(fabsf(__fdividef(mul(k.gamma, pL), rL)));
  const float aR = sqrtf(fabsf(__fdividef(mul(k.gamma, pR), rR)));
  float SL = fminf(sub(unL, aL), sub(unR, aR));
  float SR = fmaxf(add(unL, aL), add(unR, aR));
  if (SL == SR) SL = sub(SL, k.ss_eps);
  if (SL == SR) SR = add(SR, k.ss_eps);
  const float dL = sub(SL, unL), dR = sub(SR, unR);
  float den = sub(mul(rL, dL), mul(rR, dR));
  if (den == 0.0f) den = k.den_eps;
  const float Ss = __fdividef(sub(fma(mul(rL, unL), dL, sub(pR, pL)), mul(mul(rR, unR), dR)), den);
  const float PsL = fma(mul(rL, dL), sub(Ss, unL), pL);
  const float PsR = fma(mul(rR, dR), sub(Ss, unR), pR);
  const float Ps = mul(k.half, add(PsL, PsR));
  const bool c1 = SL >= 0.0f;
  const bool c2 = (SL <= 0.0f) && (Ss >= 0.0f);
  const bool c3 = (Ss <= 0.0f) && (SR >= 0.0f);
  const bool left = c1 || c2;
  const float rK = left ? rL : rR, uK = left ? uL : uR, vK = left ? vL : vR, pK = left ? pL : pR;
  const float unK = left ? unL : unR, SK = left ? SL : SR, dK = left ? dL : dR;
  const float EK = fma(mul(k.half, rK), fma(uK, uK, mul(vK, vK)), mul(pK, k.inv_gm1));
  const float ruK = mul(rK, uK), rvK = mul(rK, vK);
  const float FK0 = mul(rK, unK), FK1 = fma(pK, nx, mul(ruK, unK)), FK2 = fma(pK, ny, mul(rvK, unK));
  const float FK3 = mul(add(EK, pK), unK);
  if (left ? !c1 : c3) {
    const float inv = __fdividef(1.0f, sub(SK, Ss));
    const float rs = mul(mul(rK, dK), inv);
    const float Us3 = mul(fma(Ps, Ss, sub(mul(dK, EK), mul(pK, unK))), inv);
    const float utK = fma(uK, tx, mul(vK, ty));
    const float Us1 = mul(rs, fma(Ss, nx, mul(utK, tx))), Us2 = mul(rs, fma(Ss, ny, mul(utK, ty)));
    F[0] = fma(SK, sub(rs, rK), FK0);
    F[1] = fma(SK, sub(Us1, ruK), FK1);
    F[2] = fma(SK, sub(Us2, rvK), FK2);
    F[3] = fma(SK, sub(Us3, EK), FK3);
  } else {
    F[0] = FK0; F[1] = FK1; F[2] = FK2; F[3] = FK3;
  }
}
// the canonical flux of a face through the cell's edge of outward normal n:
// evaluated from the face's owner (the lower cell), negated on the other side
__device__ __forceinline__ void face_flux(const float qOwn[4], const float qOther[4], float nx, float ny,
                                          bool other_owns, const Consts<float>& k, float F[4]) {
  if (other_owns) {
    hllc(qOther, qOwn, -nx, -ny, k, F);
    F[0] = -F[0]; F[1] = -F[1]; F[2] = -F[2]; F[3] = -F[3];
  } else {
    hllc(qOwn, qOther, nx, ny, k, F);
  }
}
// sum_k s_k F_k in slot order: face k's term added to acc
__device__ __forceinline__ void accumulate(int k, float sk, const float F[4], float acc[4]) {
  if (k == 0) { acc[0] = mul(sk, F[0]); acc[1] = mul(sk, F[1]); acc[2] = mul(sk, F[2]); acc[3] = mul(sk, F[3]); }
  else { acc[0] = fma(sk, F[0], acc[0]); acc[1] = fma(sk, F[1], acc[1]); acc[2] = fma(sk, F[2], acc[2]); acc[3] = fma(sk, F[3], acc[3]); }
}
// euler_solver.py:602-643: residual acc / area - sponge and the stage update
template <int STAGE>
__device__ __forceinline__ float4 cell_update(const float acc[4], float area, float sig, const float4& inlet,
                                              const float4& Wc, const float4& W0, float dt, float half,
                                              float* R0_out) {
  const float R0 = sub(__fdividef(acc[0], area), mul(sig, sub(inlet.x, Wc.x)));
  const float R1 = sub(__fdividef(acc[1], area), mul(sig, sub(inlet.y, Wc.y)));
  const float R2 = sub(__fdividef(acc[2], area), mul(sig, sub(inlet.z, Wc.z)));
  const float R3 = sub(__fdividef(acc[3], area), mul(sig, sub(inlet.w, Wc.w)));
  *R0_out = R0;
  const float m = -dt;
  if (STAGE == ST_FIRST) return make_float4(fma(m, R0, Wc.x), fma(m, R1, Wc.y), fma(m, R2, Wc.z), fma(m, R3, Wc.w));
  if (STAGE == ST_SRK2_SECOND)
    return make_float4(mul(half, fma(m, R0, add(W0.x, Wc.x))), mul(half, fma(m, R1, add(W0.y, Wc.y))),
                       mul(half, fma(m, R2, add(W0.z, Wc.z))), mul(half, fma(m, R3, add(W0.w, Wc.w))));
  return make_float4(mul(half, add(fma(m, R0, W0.x), Wc.x)), mul(half, add(fma(m, R1, W0.y), Wc.y)),
                     mul(half, add(fma(m, R2, W0.z), Wc.z)), mul(half, add(fma(m, R3, W0.w), Wc.w)));
}
}  // namespace xr

// euler_solver.py:602-628 residual = sum_k F_k s_k / area - sponge (helper.py:262-295),
// then the stage update of :630-653.
template <typename T, bool FAST, int FLUX, bool MUSCL, int STAGE, bool LOCALDT, int MINB = 0>
__global__ void __launch_bounds__(256, (kMinBlocks<T, FAST, MINB, ESR_K2_MINB>)) k_flux(const BlockMap<T> bm,
                                              const V4<T>* __restrict__ Win, const V4<T>* __restrict__ Wbase,
                                              V4<T>* __restrict__ Wout, const V4<T>* __restrict__ FV,
                                              long long total, Cases<T> cs, Consts<T> kc, int pos,
                                              const T* __restrict__ dt_local, T* __restrict__ res_out) {
  Seg<T> s;
  int first;
  block_origin(bm, s, first);
  int c, b;
  if (!item_slot(s, first + threadIdx.x, c, b)) return;
  const int g = s.case0 + b;
  if (!cs.active[g] || cs.step[g] + pos >= cs.nmax[g]) return;
  const long long gi = s.off + (long long)c * s.B + b;
  const V4<T> Wc = Win[gi];
  const int4 nb = __ldg(s.nbr + c);
  const int nbk[3] = {nb.x, nb.y, nb.z};
  const V4<T> inlet = cs.inlet[g];
  T gk[12];   // normals, face lengths, area, blend (groups 0-2)
  geo_groups<T, 3>(s, c, 0, gk);
  if constexpr (kFastPath<T, FAST> && MUSCL && FLUX == 0) {
    // fast float32 HLLC + MUSCL: canonical face fluxes and the cell update
    // rounded exactly as K2 by patches rounds them
    float acc[4];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int kind = slot_kind(nb.w, k);
      const float nx = gk[G_N0X + 2 * k], ny = gk[G_N0Y + 2 * k];
      const float4 fl = FV[(long long)k * total + gi];
      const float qL[4] = {fl.x, fl.y, fl.z, fl.w};
      float qR[4];
      if (kind == K_INTERIOR) {
        const float4 fr = FV[(long long)slot_opp(nb.w, k) * total + s.off + (long long)nbk[k] * s.B + b];
        qR[0] = fr.x; qR[1] = fr.y; qR[2] = fr.z; qR[3] = fr.w;
      } else {
        xr::ghost_prim(kind, Wc, nx, ny, inlet, kc, qR);
      }
      float F[4];
      xr::face_flux(qL, qR, nx, ny, kind == K_INTERIOR && nbk[k] < c, kc, F);
      xr::accumulate(k, gk[G_S0 + k], F, acc);
    }
    const float sig = xr::mul(cs.strength[g], gk[G_BLEND3]);
    const float dt = LOCALDT ? dt_local[gi] : cs.dt[g];
    const float4 W0 = (STAGE == ST_FIRST) ? Wc : Wbase[gi];
    float R0;
    const float4 o = xr::cell_update<STAGE>(acc, gk[G_AREA], sig, inlet, Wc, W0, dt, kc.half, &R0);
    if (STAGE == ST_FIRST && res_out != nullptr) res_out[gi] = R0;
    Wout[gi] = o;
  } else {
    T acc[4];
  #pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int kind = slot_kind(nb.w, k);
      const T nx = gk[G_N0X + 2 * k], ny = gk[G_N0Y + 2 * k];
      V4<T> WL, WR;
      T PL[4], PR[4];
      if (MUSCL) {
        const V4<T> fl = FV[(long long)k * total + gi];
        T qL[4] = {fl.x, fl.y, fl.z, fl.w};
        T qR[4];
        if (kind == K_INTERIOR) {
          const V4<T> fr = FV[(long long)slot_opp(nb.w, k) * total + s.off + (long long)nbk[k] * s.B + b];
          qR[0] = fr.x; qR[1] = fr.y; qR[2] = fr.z; qR[3] = fr.w;
        } else {
          prim<T, FAST>(ghost_cons<T, FAST>(kind, Wc, nx, ny, inlet, kc), kc.gm1, kc.half, qR);
        }
        if constexpr (kFastPath<T, FAST>) {
          // float32: the face primitives are used as reconstructed (the
          // reference converts them to conserved and back, a rounding-level
          // step); HLLC forms the conserved state of the selected side itself
  #pragma unroll
          for (int v = 0; v < 4; ++v) { PL[v] = qL[v]; PR[v] = qR[v]; }
          if (FLUX != 0) {
            WL = cons<T, FAST>(qL, kc.gm1, kc.inv_gm1, kc.half);
            WR = cons<T, FAST>(qR, kc.gm1, kc.inv_gm1, kc.half);
          }
        } else {
          WL = cons<T, FAST>(qL, kc.gm1, kc.inv_gm1, kc.half);
          WR = cons<T, FAST>(qR, kc.gm1, kc.inv_gm1, kc.half);
          prim<T, FAST>(WL, kc.gm1, kc.half, PL);
          prim<T, FAST>(WR, kc.gm1, kc.half, PR);
        }
      } else {
        WL = Wc;
        WR = (kind == K_INTERIOR) ? Win[s.off + (long long)nbk[k] * s.B + b] : ghost_cons<T, FAST>(kind, Wc, nx, ny, inlet, kc);
        prim<T, FAST>(WL, kc.gm1, kc.half, PL);
        prim<T, FAST>(WR, kc.gm1, kc.half, PR);
      }
      T F[4];
      if (FLUX == 0) {
        hllc<T, FAST>(WL, PL, WR, PR, nx, ny, kc, F);
      } else {
        rusanov<T, FAST>(WL, PL, WR, PR, nx, ny, kc, F);
      }
      const T sk = gk[G_S0 + k];
      if (k == 0) { acc[0] = sk * F[0]; acc[1] = sk * F[1]; acc[2] = sk * F[2]; acc[3] = sk * F[3]; }
      else { acc[0] = acc[0] + sk * F[0]; acc[1] = acc[1] + sk * F[1]; acc[2] = acc[2] + sk * F[2]; acc[3] = acc[3] + sk * F[3]; }
    }
    const T area = gk[G_AREA];
    const T sig = cs.strength[g] * gk[G_BLEND3];
    const T R0 = dv<T, FAST>(acc[0], area) - sig * (inlet.x - Wc.x);
    const T R1 = dv<T, FAST>(acc[1], area) - sig * (inlet.y - Wc.y);
    const T R2 = dv<T, FAST>(acc[2], area) - sig * (inlet.z - Wc.z);
    const T R3 = dv<T, FAST>(acc[3], area) - sig * (inlet.w - Wc.w);
    const T dt = LOCALDT ? dt_local[gi] : cs.dt[g];
    // density residual of the state the step starts from (density-L2 stop rule)
    if (STAGE == ST_FIRST && res_out != nullptr) res_out[gi] = R0;
    V4<T> o;
    if (STAGE == ST_FIRST) {
      o = mk4<T>(Wc.x - dt * R0, Wc.y - dt * R1, Wc.z - dt * R2, Wc.w - dt * R3);
    } else if (STAGE == ST_SRK2_SECOND) {
      const V4<T> W0 = Wbase[gi];
      o = mk4<T>(kc.half * (W0.x + Wc.x - dt * R0), kc.half * (W0.y + Wc.y - dt * R1),
                 kc.half * (W0.z + Wc.z - dt * R2), kc.half * (W0.w + Wc.w - dt * R3));
    } else {
      const V4<T> W0 = Wbase[gi];
      o = mk4<T>(kc.half * (W0.x - dt * R0 + Wc.x), kc.half * (W0.y - dt * R1 + Wc.y),
                 kc.half * (W0.z - dt * R2 + Wc.z), kc.half * (W0.w - dt * R3 + Wc.w));
    }
    Wout[gi] = o;
  }
}

// ----------------------------------------------------- K2 by patches (float32)
// The face-flux form of K2 for batched float32 HLLC + MUSCL solves: one block
// per (patch of <= kPatchCells cells, group of 32 case slots), one warp per
// cell at a time with its lanes over the 32 slots. Phase 0 copies the face
// states of the patch's cells into shared memory (asynchronous 16-byte
// copies, all issued before any is waited for). Phase 1 evaluates every
// face of the patch's cells once: an inner face (both cells in the patch) by
// its owner, the lower cell, from the two face states in shared memory,
// storing F and -F over them for both cells; a face to a cell outside the
// patch (the neighbour's face state read from global memory) and a boundary
// face by the cell itself (the canonical flux, from the owner's side). Phase 2 forms each
// cell's residual sum_k s_k F_k in slot order from shared memory (a
// deterministic cell-owned sum, no atomics), then the sponge and the stage
// update as k_flux. The fluxes equal k_flux's bit for bit.
#ifndef ESR_PATCH_MINB
#define ESR_PATCH_MINB 5
#endif
#ifndef ESR_PATCH_MINB_ALT
#define ESR_PATCH_MINB_ALT 6
#endif
#ifndef ESR_PATCH_WARPS
#define ESR_PATCH_WARPS 8
#endif
constexpr int kPatchWarps = ESR_PATCH_WARPS;

// 16-byte asynchronous global -> shared copy (zero-filled when !valid; the
// source address is read only when valid)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int STAGE, bool LOCALDT, int MINB = ESR_PATCH_MINB>
__global__ void __launch_bounds__(32 * kPatchWarps, MINB) k_flux_patch(const Seg<float>* __restrict__ segs,
                                                                  const int4* __restrict__ pblk,
                                                                  const float4* __restrict__ Win,
                                                                  const float4* __restrict__ Wbase,
                                                                  float4* __restrict__ Wout,
                                                                  const float4* __restrict__ FV, long long total,
                                                                  Cases<float> cs, Consts<float> kc, int pos,
                                                                  const float* __restrict__ dt_local,
                                                                  float* __restrict__ res_out) {
  // the patch's face states, then in place its signed face fluxes (1.5 KB per cell)
  __shared__ float4 G[kPatchCells][3][32];
  const int4 pb = pblk[blockIdx.x];          // segment, patch, first slot
  const Seg<float> s = segs[pb.x];
  const int c0 = s.patch_start[pb.y], c1 = s.patch_start[pb.y + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b = pb.z + lane;
  const bool in_seg = b < s.B;
  const int g = s.case0 + (in_seg ? b : 0);
  const bool live = in_seg && cs.active[g] && cs.step[g] + pos < cs.nmax[g];
  if (!__syncthreads_or(live)) return;        // every slot of the group idle
  const float4 inlet = cs.inlet[g];
  // Phase 0: every face state of the patch's cells (this block's 32 slots)
  // into G by asynchronous copies, all in flight at once.
  for (int lc = warp; lc < c1 - c0; lc += kPatchWarps) {
    const long long gi = s.off + (long long)(c0 + lc) * s.B + b;
#pragma unroll
    for (int k = 0; k < 3; ++k) cp_async16(&G[lc][k][lane], FV + (long long)k * total + (in_seg ? gi : 0), in_seg);
  }
  cp_async_wait_all();
  __syncthreads();
  // Phase 1. Each slot G[cell][face] is read and then overwritten by exactly
  // one evaluation, that of the face's owner (an inner face's other cell
  // skips it), so the fluxes can replace the face states in place.
  for (int lc = warp; lc < c1 - c0; lc += kPatchWarps) {
    const int c = c0 + lc;
    const long long gi = s.off + (long long)c * s.B + b;
    const int4 nb = __ldg(s.nbr + c);
    const int nbk[3] = {nb.x, nb.y, nb.z};
    float gk[12];
    geo_groups<float, 3>(s, c, 0, gk);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int kind = slot_kind(nb.w, k);
      const float nx = gk[G_N0X + 2 * k], ny = gk[G_N0Y + 2 * k];
      const int j = nbk[k];
      const bool inner = kind == K_INTERIOR && j >= c0 && j < c1;
      if (inner && j < c) continue;   // the owner, inside the patch, stores this one
      const int ko = slot_opp(nb.w, k);
      const float4 fl = G[lc][k][lane];
      const float qL[4] = {fl.x, fl.y, fl.z, fl.w};
      float qR[4] = {0.f, 0.f, 0.f, 0.f};
      if (inner) {
        const float4 fr = G[j - c0][ko][lane];
        qR[0] = fr.x; qR[1] = fr.y; qR[2] = fr.z; qR[3] = fr.w;
      } else if (in_seg) {
        if (kind == K_INTERIOR) {
          const float4 fr = FV[(long long)ko * total + s.off + (long long)j * s.B + b];
          qR[0] = fr.x; qR[1] = fr.y; qR[2] = fr.z; qR[3] = fr.w;
        } else {
          xr::ghost_prim(kind, Win[gi], nx, ny, inlet, kc, qR);
        }
      }
      float F[4];
      xr::face_flux(qL, qR, nx, ny, kind == K_INTERIOR && j < c, kc, F);   // owner outside: its side, negated
      G[lc][k][lane] = make_float4(F[0], F[1], F[2], F[3]);
      if (inner) G[j - c0][ko][lane] = make_float4(-F[0], -F[1], -F[2], -F[3]);
    }
  }
  __syncthreads();
  if (!live) return;
  for (int lc = warp; lc < c1 - c0; lc += kPatchWarps) {
    const int c = c0 + lc;
    const long long gi = s.off + (long long)c * s.B + b;
    const float4 Wc = Win[gi];
    float gk[12];
    geo_groups<float, 3>(s, c, 0, gk);
    float acc[4];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 f = G[lc][k][lane];
      const float F[4] = {f.x, f.y, f.z, f.w};
      xr::accumulate(k, gk[G_S0 + k], F, acc);
    }
    const float sig = xr::mul(cs.strength[g], gk[G_BLEND3]);
    const float dt = LOCALDT ? dt_local[gi] : cs.dt[g];
    const float4 W0 = (STAGE == ST_FIRST) ? Wc : Wbase[gi];
    float R0;
    const float4 o = xr::cell_update<STAGE>(acc, gk[G_AREA], sig, inlet, Wc, W0, dt, kc.half, &R0);
    if (STAGE == ST_FIRST && res_out != nullptr) res_out[gi] = R0;
    Wout[gi] = o;
  }
}

// copy a stage result back into the state for live slots (explicit Euler)
template <typename T>
__global__ void k_commit(const Seg<T>* __restrict__ segs, const int2* __restrict__ blk, const V4<T>* __restrict__ src,
                         V4<T>* __restrict__ dst, Cases<T> cs, int pos) {
  const int2 bt = blk[blockIdx.x];
  const Seg<T> s = segs[bt.x];
  const int item = bt.y + threadIdx.x;
  if (item >= s.n_cells * s.B) return;
  const int c = cell_of(s, item);
  const int g = s.case0 + (item - c * s.B);
  if (!cs.active[g] || cs.step[g] + pos >= cs.nmax[g]) return;
  dst[s.off + item] = src[s.off + item];
}

// ------------------------------------------------------ per-case reductions
enum RedOp { RED_NORM = 0, RED_DTMIN = 1, RED_ENTROPY = 2, RED_DIFF = 3, RED_RESSQ = 4 };

struct CaseMap {             // global slot -> (segment, slot)
  const int* seg;
  const int* slot;
};

// Block (chunk, case) reduces a fixed cell range of one case; partials are
// combined in a fixed order by the consumer, so results are bitwise
// reproducible. RED_NORM: sum |W - Wref|^2, sum |Wref|^2 and Wref <- W
// (euler/main.py:150-152); RED_DTMIN: min_i area/sum_k (c+|u.n|) s
// (helper.py:8-18); RED_ENTROPY: sum rho log(p/rho^g) area/(g-1)
// (helper.py:48-55,312-315); RED_DIFF: sum |A - B|^2, sum |B|^2 (probe).
template <typename T, int OP, bool FAST = (sizeof(T) == 4)>
__global__ void __launch_bounds__(256) k_case_reduce(const Seg<T>* __restrict__ segs, CaseMap cm,
                                                     const V4<T>* __restrict__ W, V4<T>* __restrict__ Wref,
                                                     const int* __restrict__ due, int chunk_cells,
                                                     double2* __restrict__ partial, int n_chunks, Consts<T> kc) {
  const int g = blockIdx.y;
  const int chunk = blockIdx.x;
  if (due != nullptr && !due[g]) return;
  const int si = cm.seg[g];
  const Seg<T> s = segs[si];
  const int b = cm.slot[g];
  const int c0 = chunk * chunk_cells;
  const int c1 = min(s.n_cells, c0 + chunk_cells);
  double a0 = (OP == RED_DTMIN) ? 1e300 : 0.0, a1 = 0.0;
  for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    const long long gi = s.off + (long long)c * s.B + b;
    const V4<T> w = W[gi];
    if (OP == RED_NORM || OP == RED_DIFF) {
      const V4<T> r = Wref[gi];
      const double d0 = (double)w.x - (double)r.x, d1 = (double)w.y - (double)r.y;
      const double d2 = (double)w.z - (double)r.z, d3 = (double)w.w - (double)r.w;
      a0 += d0 * d0 + d1 * d1 + d2 * d2 + d3 * d3;
      a1 += (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z + (double)r.w * r.w;
      if (OP == RED_NORM) Wref[gi] = w;
    } else if (OP == RED_DTMIN) {
      T P[4];
      prim<T, FAST>(w, kc.gm1, kc.half, P);
      const T cel = sqrt(fabs(kc.gamma * P[3] / P[0]));
      T lam = T(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const T un = P[1] * geo(s, G_N0X + 2 * k, c) + P[2] * geo(s, G_N0Y + 2 * k, c);
        const T term = (cel + fabs(un)) * geo(s, G_S0 + k, c);
        lam = (k == 0) ? term : lam + term;
      }
      const T d = geo(s, G_AREA, c) / lam;
      a0 = fmin(a0, (double)d);
    } else if (OP == RED_RESSQ) {   // Wref carries the density residual array
      const double r = (double)((const T*)Wref)[gi];
      a0 += r * r;
      a1 += 1.0;
    } else {  // entropy
      const T r = w.x, u = w.y / r, v = w.z / r;
      const T p = (w.w - kc.half * r * (u * u + v * v)) * kc.gm1;
      const T sv = log(p / pow(r, kc.gamma));
      a0 += (double)(r * sv * geo(s, G_AREA, c) / kc.gm1);
    }
  }
  // fixed-shape block reduction
  __shared__ double sh0[256], sh1[256];
  sh0[threadIdx.x] = a0;
  sh1[threadIdx.x] = a1;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      if (OP == RED_DTMIN) sh0[threadIdx.x] = fmin(sh0[threadIdx.x], sh0[threadIdx.x + w]);
      else { sh0[threadIdx.x] += sh0[threadIdx.x + w]; sh1[threadIdx.x] += sh1[threadIdx.x + w]; }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[(size_t)g * n_chunks + chunk] = make_double2(sh0[0], sh1[0]);
}

// ---------------------------------------------------------- case bookkeeping
struct CaseCtl {             // mutable per-slot control words (device)
  int* active;
  int* step;
  int* nmax;
  int* ref_step;
  int* streak;
  int* streak_start;
  int* stopping_step;
  int* status;
  int* due;
  double* last_rel;
  long long* t_start;        // globaltimer at the case start (ns)
  long long* t_end;
  // engineering criterion (euler/main.py:66-113,160-171)
  const int* eng_track;
  const int* eng_patience;
  const double4* eng_t;      // target cd, target cl, |cd| tolerance, |cl| tolerance
  int* eng_streak;
  int* eng_start;
  int* eng_stop;
  int* eng_stopping;
  const double* forces;      // cd, cl per slot at the current check
  const double* thr;         // per-slot stop-rule threshold, <= 0: the solver's
};

// step-0 engineering state of freshly filled slots (euler/main.py:107-111)
static __global__ void k_eng_init(CaseCtl cc, const int* __restrict__ fill, int n_slots) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots || !fill[g]) return;
  int ok = 0;
  if (cc.eng_track[g]) {
    const double4 t = cc.eng_t[g];
    ok = fabs(cc.forces[2 * g] - t.x) <= t.z && fabs(cc.forces[2 * g + 1] - t.y) <= t.w;
  }
  cc.eng_streak[g] = ok;
  cc.eng_start[g] = 0;
  cc.eng_stop[g] = 0;
  cc.eng_stopping[g] = cc.nmax[g];
}

// Which slots need a stop-rule check after `pos` steps of the chunk.
static __global__ void k_mark_due(CaseCtl cc, int n_slots, int pos, int check_every) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots) return;
  int d = 0;
  if (cc.active[g]) {
    const int done = min(cc.step[g] + pos, cc.nmax[g]);
    d = (done > cc.ref_step[g]) && ((done % check_every) == 0 || done >= cc.nmax[g]);
  }
  cc.due[g] = d;
}

__device__ __forceinline__ long long globaltimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// euler/main.py:147-158: rel, streak, confirmation and the stopping step.
// STOP_RULE 0: rel = ||dW|| / (block * (||Wref|| + 1e-16)); 1: density-residual RMS
static __global__ void k_check(CaseCtl cc, int n_slots, int pos, const double2* __restrict__ partial, int n_chunks,
                        const int* __restrict__ ncells, double threshold, int patience, int stop_rule,
                        int check_every) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots || !cc.due[g]) return;
  double s0 = 0.0, s1 = 0.0;
  for (int i = 0; i < n_chunks; ++i) {
    const double2 p = partial[(size_t)g * n_chunks + i];
    s0 += p.x;
    s1 += p.y;
  }
  const int done = min(cc.step[g] + pos, cc.nmax[g]);
  const int block = max(1, done - cc.ref_step[g]);
  double rel;
  if (stop_rule == 0) rel = sqrt(s0) / ((double)block * (sqrt(s1) + 1e-16));
  else rel = sqrt(s0 / (double)ncells[g]);
  cc.last_rel[g] = rel;
  const bool finite = isfinite(s0) && isfinite(s1);
  const double th = cc.thr[g] > 0.0 ? cc.thr[g] : threshold;
  const bool under = rel <= th;
  const int streak = cc.streak[g];
  const int nstreak = under ? streak + 1 : 0;
  if (under && streak == 0) cc.streak_start[g] = done;
  cc.streak[g] = nstreak;
  cc.ref_step[g] = done;
  int st = 0;
  if (!finite) st = 4;
  else if (stop_rule != 2 && nstreak >= patience) st = 2;
  else if (done >= cc.nmax[g]) st = 3;
  bool eng_under = false;
  if (cc.eng_track[g]) {
    const double4 t = cc.eng_t[g];
    eng_under = fabs(cc.forces[2 * g] - t.x) <= t.z && fabs(cc.forces[2 * g + 1] - t.y) <= t.w;
    const int es = cc.eng_streak[g];
    const int nes = eng_under ? es + 1 : 0;
    if (eng_under && es == 0) cc.eng_start[g] = done;
    cc.eng_streak[g] = nes;
    if (nes >= cc.eng_patience[g] && !cc.eng_stop[g]) {
      cc.eng_stop[g] = 1;
      cc.eng_stopping[g] = cc.eng_start[g];
      if (stop_rule == 2 && finite) {   // the criterion itself ends the case
        st = 2;
        cc.streak_start[g] = cc.eng_start[g];
      }
    }
    // The reference keeps checking the frozen field after the stop rule
    // fires until step N: the criterion can still confirm on that field.
    if (st == 2 && !cc.eng_stop[g] && eng_under) {
      const int ce = max(1, check_every);
      const int N = cc.nmax[g];
      const int remaining = done >= N ? 0 : N / ce - done / ce + ((N % ce) ? 1 : 0);
      if (nes + remaining >= cc.eng_patience[g]) {
        cc.eng_stop[g] = 1;
        cc.eng_stopping[g] = cc.eng_start[g];
      }
    }
  }
  if (st) {
    cc.status[g] = st;
    cc.stopping_step[g] = (st == 2) ? cc.streak_start[g] : cc.nmax[g];
    cc.step[g] = done;
    cc.active[g] = 0;
    cc.t_end[g] = globaltimer();
  }
}

// chunk end without checks: every live slot advanced `len` steps
static __global__ void k_advance(CaseCtl cc, int n_slots, int len, int stop_at_nmax) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots || !cc.active[g]) return;
  const int done = min(cc.step[g] + len, cc.nmax[g]);
  cc.step[g] = done;
  if (stop_at_nmax && done >= cc.nmax[g] && cc.status[g] == 1) {
    cc.status[g] = 3;
    cc.stopping_step[g] = cc.nmax[g];
    cc.active[g] = 0;
    cc.t_end[g] = globaltimer();
  }
}

// dt of freshly (re)filled slots from the RED_DTMIN partials: dt = CFL * min,
// N = int(tf / dt) + 1 in the state precision (euler/main.py:121-122)
template <typename T>
__global__ void k_dt_finish(const int* __restrict__ fill, int n_slots, const double2* __restrict__ partial,
                            int n_chunks, const double* __restrict__ cfl, const double* __restrict__ tf,
                            const long long* __restrict__ max_steps, T* __restrict__ dt, CaseCtl cc, int local_mode) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots || !fill[g]) return;
  double m = 1e300;
  for (int i = 0; i < n_chunks; ++i) m = fmin(m, partial[(size_t)g * n_chunks + i].x);
  const T d = (T)m * (T)cfl[g];
  long long n;
  if (local_mode) {
    dt[g] = (T)cfl[g];
    n = max_steps[g] > 0 ? max_steps[g] : (long long)((T)tf[g] / d) + 1;
  } else {
    dt[g] = d;
    n = (long long)((T)tf[g] / d) + 1;
  }
  if (max_steps[g] > 0 && n > max_steps[g]) n = max_steps[g];
  if (!(n >= 1)) n = 1;
  if (n > 2000000000LL) n = 2000000000LL;
  cc.nmax[g] = (int)n;
  cc.t_start[g] = globaltimer();
}

// ------------------------------------------------- device-side case queue
// A batch of cases is uploaded once; every chunk of steps ends with a refill
// sequence inside the same CUDA graph: slots whose case stopped write the
// case's result record (and final state), then each mesh's free slots take
// the next queued cases of that mesh in slot order, their state is set from
// the freestream or an uploaded warm start, and dt, N and the step-0
// engineering state are computed. The host only polls the done counter.
template <typename T>
struct Queue {
  int n_meshes;
  const int* qlist;            // case ids grouped by mesh, in submission order
  const int* qoff;             // n_meshes + 1 offsets into qlist
  int* qhead;                  // per mesh: next queue position
  int* slot_case;              // per slot: running case id or -1
  int* retiring;               // per slot scratch flag
  // per case parameters
  const V4<T>* c_inlet;
  const T* c_strength;
  const double* c_cfl;
  const double* c_tf;
  const long long* c_max_steps;
  const double* c_qref;
  const int* c_eng_track;
  const int* c_eng_pat;
  const double4* c_eng_t;
  const double* c_thr;
  const double* init;          // warm-start rows (caller cell order), or null
  const long long* init_off;   // per case first row in `init`, -1 = freestream
  // per case results
  int* r_status;
  int* r_stop;
  int* r_steps;
  int* r_nmax;
  double* r_dt;
  double* r_rel;
  double* r_cd;
  double* r_cl;
  double* r_time;
  int* r_eng_conv;
  int* r_eng_stop;
  double* r_probe;             // one-step residual of the final state
  double* out;                 // final states (caller order) or null
  const long long* out_off;    // per case first row in `out`
  int* n_done;
};

// per-slot writable parameters that the queue fills
template <typename T>
struct SlotParams {
  T* dt;
  V4<T>* inlet;
  T* strength;
  double* cfl;
  double* tf;
  long long* max_steps;
  double* qref;
  int* eng_track;
  int* eng_pat;
  double4* eng_t;
  double* thr;
};

static __global__ void k_mark_retiring(const int* __restrict__ status, int n_slots, int* __restrict__ slot_case,
                                       int* __restrict__ retiring) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots) return;
  retiring[g] = (slot_case[g] >= 0 && status[g] >= 2) ? 1 : 0;
}

// result record of every retiring slot's case (forces already computed)
template <typename T>
__global__ void k_retire(CaseCtl cc, Queue<T> q, const T* __restrict__ dt, const double* __restrict__ forces,
                         int n_slots, int local_mode) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots || !q.retiring[g]) return;
  const int c = q.slot_case[g];
  const int st = cc.status[g];
  q.r_status[c] = st;
  q.r_stop[c] = cc.stopping_step[g];
  q.r_steps[c] = cc.step[g];
  q.r_nmax[c] = cc.nmax[g];
  q.r_dt[c] = local_mode ? 0.0 : (double)dt[g];
  q.r_rel[c] = cc.last_rel[g];
  q.r_cd[c] = forces[2 * g];
  q.r_cl[c] = forces[2 * g + 1];
  q.r_time[c] = (cc.t_end[g] > cc.t_start[g]) ? (double)(cc.t_end[g] - cc.t_start[g]) * 1e-9 : 0.0;
  const int tr = cc.eng_track[g];
  q.r_eng_conv[c] = tr ? cc.eng_stop[g] : 0;
  q.r_eng_stop[c] = tr ? (cc.eng_stop[g] ? cc.eng_stopping[g] : cc.nmax[g]) : 0;
  atomicAdd(q.n_done, 1);   // a counter only; no result depends on its order
}

// euler/main.py:228-230 for every retiring slot: ||W' - W|| / (||W|| + 1e-16)
// from the RED_DIFF partials of its probe step, summed in chunk order
template <typename T>
__global__ void k_probe_finish(Queue<T> q, const double2* __restrict__ partial, int n_chunks, int n_slots) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots || !q.retiring[g]) return;
  double s0 = 0.0, s1 = 0.0;
  for (int i = 0; i < n_chunks; ++i) {
    s0 += partial[(size_t)g * n_chunks + i].x;
    s1 += partial[(size_t)g * n_chunks + i].y;
  }
  q.r_probe[q.slot_case[g]] = sqrt(s0) / (sqrt(s1) + 1e-16);
}

// final state of retiring slots into the output rows (caller cell order)
template <typename T>
__global__ void k_retire_states(const Seg<T>* __restrict__ segs, CaseMap cm, Queue<T> q, const V4<T>* __restrict__ W,
                                const int* __restrict__ const* inv_of_seg) {
  const int g = blockIdx.y;
  if (!q.retiring[g] || q.out == nullptr) return;
  const Seg<T> s = segs[cm.seg[g]];
  const int b = cm.slot[g];
  const int* inv = inv_of_seg[cm.seg[g]];
  const long long base = q.out_off[q.slot_case[g]];
  for (int cc = blockIdx.x * blockDim.x + threadIdx.x; cc < s.n_cells; cc += gridDim.x * blockDim.x) {
    const V4<T> w = W[s.off + (long long)inv[cc] * s.B + b];
    double* r = q.out + 4 * (base + cc);
    r[0] = (double)w.x; r[1] = (double)w.y; r[2] = (double)w.z; r[3] = (double)w.w;
  }
}

// one thread per mesh: free slots take the next queued cases, in slot order
template <typename T>
__global__ void k_assign(const Seg<T>* __restrict__ segs, int n_segs, Queue<T> q, SlotParams<T> sp, CaseCtl cc,
                         int* __restrict__ fill) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n_segs) return;
  const Seg<T> s = segs[m];
  for (int b = 0; b < s.B; ++b) {
    const int g = s.case0 + b;
    fill[g] = 0;
    if (q.slot_case[g] >= 0 && !q.retiring[g]) continue;   // still running
    q.retiring[g] = 0;
    if (q.qhead[m] >= q.qoff[m + 1] - q.qoff[m]) {
      q.slot_case[g] = -1;
      cc.active[g] = 0;
      cc.status[g] = 0;
      continue;
    }
    const int c = q.qlist[q.qoff[m] + q.qhead[m]];
    q.qhead[m] += 1;
    q.slot_case[g] = c;
    fill[g] = 1;
    sp.inlet[g] = q.c_inlet[c];
    sp.strength[g] = q.c_strength[c];
    sp.cfl[g] = q.c_cfl[c];
    sp.tf[g] = q.c_tf[c];
    sp.max_steps[g] = q.c_max_steps[c];
    sp.qref[g] = q.c_qref[c];
    sp.eng_track[g] = q.c_eng_track[c];
    sp.eng_pat[g] = q.c_eng_pat[c];
    sp.eng_t[g] = q.c_eng_t[c];
    sp.thr[g] = q.c_thr[c];
    cc.step[g] = 0;
    cc.ref_step[g] = 0;
    cc.streak[g] = 0;
    cc.streak_start[g] = 0;
    cc.stopping_step[g] = 0;
    cc.due[g] = 0;
    cc.status[g] = 1;
    cc.active[g] = 1;
    cc.last_rel[g] = INFINITY;
  }
}

// initial state of the slots just filled: warm-start rows or freestream
template <typename T>
__global__ void k_fill_slots(const Seg<T>* __restrict__ segs, CaseMap cm, Queue<T> q, const int* __restrict__ fill,
                             const int* __restrict__ const* perm_of_seg, V4<T>* __restrict__ W,
                             V4<T>* __restrict__ Wref) {
  const int g = blockIdx.y;
  if (!fill[g]) return;
  const Seg<T> s = segs[cm.seg[g]];
  const int b = cm.slot[g];
  const int c = q.slot_case[g];
  const long long off = (q.init != nullptr) ? q.init_off[c] : -1;
  const int* perm = perm_of_seg[cm.seg[g]];
  const V4<T> inl = q.c_inlet[c];
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < s.n_cells; cell += gridDim.x * blockDim.x) {
    V4<T> w = inl;
    if (off >= 0) {
      const double* r = q.init + 4 * (off + perm[cell]);
      w = mk4<T>((T)r[0], (T)r[1], (T)r[2], (T)r[3]);
    }
    const long long gi = s.off + (long long)cell * s.B + b;
    W[gi] = w;
    Wref[gi] = w;
  }
}

// per-slot start of a case (esr_set_cases): parameters and reset counters
template <typename T>
struct SlotInit {
  V4<T> inlet;
  double cfl, tf, qref, thr;
  long long max_steps;
  double4 eng_t;
  T strength;
  int slot, eng_track, eng_pat;
};

template <typename T>
__global__ void k_init_slots(const SlotInit<T>* __restrict__ si, int n, SlotParams<T> sp, CaseCtl cc,
                             int* __restrict__ fill) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SlotInit<T> x = si[i];
  const int g = x.slot;
  sp.inlet[g] = x.inlet;
  sp.strength[g] = x.strength;
  sp.cfl[g] = x.cfl;
  sp.tf[g] = x.tf;
  sp.max_steps[g] = x.max_steps;
  sp.qref[g] = x.qref;
  sp.eng_track[g] = x.eng_track;
  sp.eng_pat[g] = x.eng_pat;
  sp.eng_t[g] = x.eng_t;
  sp.thr[g] = x.thr;
  cc.step[g] = 0;
  cc.ref_step[g] = 0;
  cc.streak[g] = 0;
  cc.streak_start[g] = 0;
  cc.stopping_step[g] = 0;
  cc.due[g] = 0;
  cc.status[g] = 1;
  cc.active[g] = 1;
  cc.last_rel[g] = INFINITY;
  fill[g] = 1;
}

// Once a mesh's queue is empty its running cases are packed into the lowest
// slots, so that warps over the freed slots (32 slots of one cell) exit at
// once in the step kernels. One thread per mesh pairs the lowest free slot
// with the highest running one; move_src[dst] = src, -1 elsewhere.
template <typename T>
__global__ void k_compact_plan(const Seg<T>* __restrict__ segs, int n_segs, Queue<T> q, int* __restrict__ move_src,
                               int4* __restrict__ live) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n_segs) return;
  const Seg<T> s = segs[m];
  for (int b = 0; b < s.B; ++b) move_src[s.case0 + b] = -1;
  if (q.qhead[m] < q.qoff[m + 1] - q.qoff[m]) {   // cases still queued: no slot is free
    live[m] = make_int4(s.B, (int)s.b_magic, s.b_shift, 0);
    return;
  }
  // after the moves the running cases fill slots 0..A-1: the step kernels walk those alone
  int running = 0;
  for (int b = 0; b < s.B; ++b) running += q.slot_case[s.case0 + b] >= 0;
  const Divider d = make_divider((unsigned)max(running, 1));
  live[m] = make_int4(running, (int)d.magic, d.shift, 0);
  int lo = 0, hi = s.B - 1;
  for (;;) {
    while (lo < hi && q.slot_case[s.case0 + lo] >= 0) ++lo;
    while (hi > lo && q.slot_case[s.case0 + hi] < 0) --hi;
    if (lo >= hi) break;
    move_src[s.case0 + lo] = s.case0 + hi;
    ++lo;
    --hi;
  }
}

// per-cell state of every moved case (grid: x over cells, y over slots)
template <typename T>
__global__ void k_compact_items(const Seg<T>* __restrict__ segs, CaseMap cm, const int* __restrict__ move_src,
                                V4<T>* __restrict__ W, V4<T>* __restrict__ Wref) {
  const int g = blockIdx.y;
  const int src = move_src[g];
  if (src < 0) return;
  const Seg<T> s = segs[cm.seg[g]];
  const int bd = cm.slot[g], bs = cm.slot[src];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < s.n_cells; c += gridDim.x * blockDim.x) {
    const long long d = s.off + (long long)c * s.B + bd, o = s.off + (long long)c * s.B + bs;
    W[d] = W[o];
    Wref[d] = Wref[o];
  }
}

// per-slot words of every moved case; the source slot is left empty
template <typename T>
__global__ void k_compact_slots(const int* __restrict__ move_src, int n_slots, Queue<T> q, SlotParams<T> sp,
                                CaseCtl cc, double* __restrict__ forces) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_slots) return;
  const int o = move_src[g];
  if (o < 0) return;
  q.slot_case[g] = q.slot_case[o];
  sp.dt[g] = sp.dt[o]; sp.inlet[g] = sp.inlet[o]; sp.strength[g] = sp.strength[o]; sp.cfl[g] = sp.cfl[o];
  sp.tf[g] = sp.tf[o]; sp.max_steps[g] = sp.max_steps[o]; sp.qref[g] = sp.qref[o];
  sp.eng_track[g] = sp.eng_track[o]; sp.eng_pat[g] = sp.eng_pat[o]; sp.eng_t[g] = sp.eng_t[o];
  sp.thr[g] = sp.thr[o];
  cc.active[g] = cc.active[o]; cc.step[g] = cc.step[o]; cc.nmax[g] = cc.nmax[o]; cc.ref_step[g] = cc.ref_step[o];
  cc.streak[g] = cc.streak[o]; cc.streak_start[g] = cc.streak_start[o]; cc.stopping_step[g] = cc.stopping_step[o];
  cc.status[g] = cc.status[o]; cc.due[g] = cc.due[o]; cc.last_rel[g] = cc.last_rel[o];
  cc.t_start[g] = cc.t_start[o]; cc.t_end[g] = cc.t_end[o];
  cc.eng_streak[g] = cc.eng_streak[o]; cc.eng_start[g] = cc.eng_start[o]; cc.eng_stop[g] = cc.eng_stop[o];
  cc.eng_stopping[g] = cc.eng_stopping[o];
  forces[2 * g] = forces[2 * o];
  forces[2 * g + 1] = forces[2 * o + 1];
  q.slot_case[o] = -1;
  cc.active[o] = 0;
  cc.status[o] = 0;
  cc.due[o] = 0;
}

// pressure force coefficients of every live-or-finished slot
// (helper.py:366-415): sum_w p(cell_w) n_w ds_w / (q_inf L_ref), p at gamma 1.4
template <typename T>
__global__ void k_forces(const Seg<T>* __restrict__ segs, CaseMap cm, const V4<T>* __restrict__ W,
                         const double* __restrict__ qref, double* __restrict__ out, Consts<T> kc,
                         const int* __restrict__ only_a, const int* __restrict__ only_b) {
  const int g = blockIdx.x;
  if ((only_a && !only_a[g]) || (only_b && !only_b[g])) return;   // optional slot filters
  const Seg<T> s = segs[cm.seg[g]];
  const int b = cm.slot[g];
  double ax = 0.0, ay = 0.0;
  for (int i = threadIdx.x; i < s.n_wall; i += blockDim.x) {
    const int c = s.wall_cell[i];
    T P[4];
    prim<T>(W[s.off + (long long)c * s.B + b], kc.gm1_14, kc.half, P);
    ax += (double)(P[3] * s.wall_nx[i] * s.wall_ds[i]);
    ay += (double)(P[3] * s.wall_ny[i] * s.wall_ds[i]);
  }
  __shared__ double sx[256], sy[256];
  sx[threadIdx.x] = ax;
  sy[threadIdx.x] = ay;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { sx[threadIdx.x] += sx[threadIdx.x + w]; sy[threadIdx.x] += sy[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * g] = sx[0] / qref[g];
    out[2 * g + 1] = sy[0] / qref[g];
  }
}

// ----------------------------------------------------------- state movers
// host-order rows (float64, or float32) -> device precision, cell c of the
// caller's order goes to renumbered cell inv[c]
template <typename T, typename S = double>
__global__ void k_scatter_state(const S* __restrict__ src, const int* __restrict__ inv, int n_cells,
                                V4<T>* __restrict__ W, V4<T>* __restrict__ Wref, long long off, int B, int b) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  const S* r = src + 4 * (size_t)c;
  const V4<T> w = mk4<T>((T)r[0], (T)r[1], (T)r[2], (T)r[3]);
  const long long gi = off + (long long)inv[c] * B + b;
  W[gi] = w;
  if (Wref) Wref[gi] = w;
}

template <typename T, typename S = double>
__global__ void k_gather_state(const V4<T>* __restrict__ W, const int* __restrict__ inv, int n_cells,
                               long long off, int B, int b, S* __restrict__ dst) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  const V4<T> w = W[off + (long long)inv[c] * B + b];
  S* r = dst + 4 * (size_t)c;
  r[0] = (S)w.x; r[1] = (S)w.y; r[2] = (S)w.z; r[3] = (S)w.w;
}

// One slot's field in a staging buffer of host rows (caller cell order):
// many slots move with one launch (grid.y = slot).
template <typename T>
struct SlotCopy {
  long long stage_row;   // first row of the slot in the staging buffer; < 0: fill with w
  const int* inv;        // caller cell -> solver cell of the slot's mesh
  long long off;         // the mesh's first item
  int n_cells, B, b, pad;
  V4<T> w;               // freestream state of a fill
};

// W = Wref = the staged rows (or the freestream) of every slot of jobs
template <typename T, typename S>
__global__ void k_scatter_slots(const S* __restrict__ stage, const SlotCopy<T>* __restrict__ jobs,
                                V4<T>* __restrict__ W, V4<T>* __restrict__ Wref) {
  const SlotCopy<T> j = jobs[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= j.n_cells) return;
  V4<T> w;
  long long gi;
  if (j.stage_row >= 0) {
    const S* r = stage + 4 * (j.stage_row + c);
    w = mk4<T>((T)r[0], (T)r[1], (T)r[2], (T)r[3]);
    gi = j.off + (long long)j.inv[c] * j.B + j.b;
  } else {
    w = j.w;
    gi = j.off + (long long)c * j.B + j.b;
  }
  W[gi] = w;
  Wref[gi] = w;
}

// the staged rows of every slot of jobs from W, in caller cell order
template <typename T, typename S>
__global__ void k_gather_slots(const V4<T>* __restrict__ W, const SlotCopy<T>* __restrict__ jobs,
                               S* __restrict__ stage) {
  const SlotCopy<T> j = jobs[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= j.n_cells) return;
  const V4<T> w = W[j.off + (long long)j.inv[c] * j.B + j.b];
  S* r = stage + 4 * (j.stage_row + c);
  r[0] = (S)w.x; r[1] = (S)w.y; r[2] = (S)w.z; r[3] = (S)w.w;
}

// every item of W set to one state (the autotuner's workload)
template <typename T>
__global__ void k_fill_uniform(V4<T>* __restrict__ W, long long n, V4<T> w) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    W[i] = w;
}

// freestream fill of a slot: W = Wref = inlet
template <typename T>
__global__ void k_fill_freestream(V4<T>* __restrict__ W, V4<T>* __restrict__ Wref, int n_cells, long long off, int B,
                                  int b, V4<T> w) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  const long long gi = off + (long long)c * B + b;
  W[gi] = w;
  Wref[gi] = w;
}

// state in the device precision, caller cell order <-> solver order
template <typename T>
__global__ void k_copy_in_device(const V4<T>* __restrict__ src, const int* __restrict__ inv, int n_cells,
                                 V4<T>* __restrict__ W, V4<T>* __restrict__ Wref, long long off, int B, int b) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  const long long gi = off + (long long)inv[c] * B + b;
  W[gi] = src[c];
  if (Wref) Wref[gi] = src[c];
}

template <typename T>
__global__ void k_copy_out_device(const V4<T>* __restrict__ W, const int* __restrict__ inv, int n_cells,
                                  long long off, int B, int b, V4<T>* __restrict__ dst) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  dst[c] = W[off + (long long)inv[c] * B + b];
}

// ------------------------------------------------------------------- IDW
// eval/core.py:135-142 with utils/metrics.py:9-14: weights from float64
// distances, float32 weighted sum over the k neighbours in order. A
// neighbour index outside [0, n_src) is never read: the row becomes NaN and
// *bad is set (the host reads it with esr_idw_status).
__device__ int g_idw_bad = 0;

static __global__ void k_idw(const float* __restrict__ src, int n_src, int n_vars, const int* __restrict__ idx,
                             const float* __restrict__ dist, int n_dst, int k, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_dst) return;
  double wsum = 0.0;
  double w[16];
  bool in_range = true;
  for (int j = 0; j < k; ++j) {
    const int q = idx[(size_t)i * k + j];
    in_range = in_range && q >= 0 && q < n_src;
    const double d = (double)dist[(size_t)i * k + j];
    w[j] = 1.0 / (d * d + 1e-12);
    wsum += w[j];
  }
  if (!in_range) {
    atomicExch(&g_idw_bad, 1);
    for (int v = 0; v < n_vars; ++v) out[(size_t)i * n_vars + v] = __int_as_float(0x7fc00000);
    return;
  }
  for (int v = 0; v < n_vars; ++v) {
    float acc = 0.0f;
    for (int j = 0; j < k; ++j) {
      const float wf = (float)(w[j] / wsum);
      acc += wf * src[(size_t)idx[(size_t)i * k + j] * n_vars + v];
    }
    out[(size_t)i * n_vars + v] = acc;
  }
}

}  // namespace esr
