// esr_layout.h -- data-layout constants shared by host and device code.
#pragma once

namespace esr {

// per-cell geometry, G_COUNT = 24 values per cell stored cell by cell
// (geo[cell * G_COUNT + field]) in groups of 4 for vector loads: groups 0-2
// are what the flux kernel reads, groups 3-5 what the reconstruction reads
enum GeoField {
  G_N0X, G_N0Y, G_N1X, G_N1Y,                 // outward unit normals
  G_N2X, G_N2Y, G_S0, G_S1,                   // ... and face lengths
  G_S2, G_AREA, G_BLEND3, G_PAD,              // cell area, sponge blend^3
  G_C0X, G_C0Y, G_C1X, G_C1Y,                 // LSQ: grad = sum_k c_k (P_k - P_c)
  G_C2X, G_C2Y, G_F0X, G_F0Y,                 // face midpoint - barycentre
  G_F1X, G_F1Y, G_F2X, G_F2Y,
  G_COUNT
};
static_assert(G_COUNT == 24, "geometry groups of 4");

// Per-cell least-squares data of the reference-fidelity float32 path, which
// forms the gradient per call as helper.py:136-153 does: offsets dx_k
// (neighbour barycentre or twice the face offset), weights 1/|dx_k|^2 and the
// 2x2 matrix A = sum_k w_k dx_k dx_k^T, all rounded as the reference's
// float32 arithmetic rounds them.
struct LsqRef {
  float w[3];
  float dx[6];      // dx_k = (dx[2k], dx[2k+1])
  float a[4];       // a00, a01, a10, a11
  float pad[3];
};
static_assert(sizeof(LsqRef) == 64, "one 64-byte record per cell");

// cells per patch of the renumbering: the face-flux kernel of batched float32
// solves exchanges the fluxes of a patch's inner faces in shared memory
// (kPatchCells x 3 x 32 lanes x 16 B per block)
#ifndef ESR_PATCH_CELLS
#define ESR_PATCH_CELLS 24
#endif
constexpr int kPatchCells = ESR_PATCH_CELLS;

// n / d without an integer divide for 0 <= n < 2^31: q = (umulhi(n, magic) +
// n) >> shift with shift = ceil(log2 d), magic = floor(2^32 (2^shift - d) / d)
// + 1 (d >= 1; magic < 2^32 because 2^(shift-1) < d)
struct Divider {
  unsigned magic;
  int shift;
};
#if defined(__CUDACC__)
__host__ __device__
#endif
inline Divider make_divider(unsigned d) {
  int l = 0;
  while ((1ull << l) < d) ++l;
  const unsigned long long m = ((1ull << 32) * ((1ull << l) - d)) / d + 1;
  return Divider{(unsigned)m, l};
}
#if defined(__CUDACC__)
__host__ __device__
#endif
inline unsigned divide(unsigned n, Divider v) {
  return (unsigned)((((unsigned long long)n * v.magic >> 32) + n) >> v.shift);
}

// slot kinds (face markers of euler/jax_fvm/src/mesh.py:47-52)
enum SlotKind { K_INTERIOR = 0, K_WALL = 2, K_INLET = 3, K_OUTLET = 4, K_SUBSONIC = 5 };

// neighbour word w: per edge slot k, bits 6k..6k+2 kind, 6k+3..6k+4 the
// neighbour's slot of the shared face
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int slot_kind(int packed, int k) { return (packed >> (6 * k)) & 7; }
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int slot_opp(int packed, int k) { return (packed >> (6 * k + 3)) & 3; }

}  // namespace esr
