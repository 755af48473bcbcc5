// Tensor-memory-accelerator (TMA) staging of the split-form face kernels' cell tiles (sm_100a).
//
// A face kernel's block stages, for each of its lines, the cells its faces read, for every primitive
// field of the state (structure of arrays: field f of cell c at f * ncells + c).  That tile is a box of
// the state seen as a (DIM + 1)-dimensional tensor (x, y[, z], field) of doubles, so one elected thread
// issues a single cp.async.bulk.tensor for all fields (and one for the time-n alpha_0 plane of the
// corrector), completing on an mbarrier, instead of every thread loading a few cells field by field.
// Cells outside the mesh (the first chunk of a line starts two cells before x = 0; lines past the last)
// are filled with zeros by the copy; the kernels never read them.
//
// The tensor maps are encoded on the host (cuTensorMapEncodeTiled, reached through the runtime's driver
// entry point, so nothing links against libcuda) once per state buffer and axis when a context is
// created, and reach the kernel as __grid_constant__ parameters.  A tiled copy needs a 16-byte aligned
// base (cudaMalloc), strides that are multiples of 16 bytes (n_x even: the host builds no map
// otherwise and the kernels load the tile themselves), an inner box extent that is a multiple of 16
// bytes (20 doubles for X faces, 16 for Y and Z faces) and an x coordinate whose byte offset is a
// multiple of 16: f0 - 2 with f0 a multiple of the X chunk (16), or the first of 16 x lines.  Every copy
// reads this GPU's own memory into its own CTA; there is no multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ecg {

// Block of the face kernel of axis AX: TF faces along AX times W lines along the fastest other axis
// (Y lines for X faces, X lines for Y and Z faces), one thread per face; the block's third coordinate
// is blockIdx.z.  Shared planes are laid out so that the linear thread order is the storage order,
// and so that a staged plane is the box a tensor copy writes: X faces [line][CP cells], Y and Z faces
// [CP cells][W lines].  A line of X faces has n_x + 1 faces, so its last chunk holds a single face:
// chunks of 16 faces keep more lanes busy than chunks of 32 on short lines (257 faces at 256^3: 94 %
// against 89 %).
#ifndef ECG_XFACE_TF
#define ECG_XFACE_TF 16
#endif
template <int AX>
struct FaceTile {
  static constexpr int TF = (AX == 0) ? ECG_XFACE_TF : 8;
  static constexpr int W = (AX == 0) ? 128 / ECG_XFACE_TF : 16;
  static constexpr int NTH = TF * W;
  // staged cells per line, from f0-2: TF + 3 are read (f0-2 .. f0+TF); X lines stage one more so a
  // staged row is a multiple of 16 bytes
  static constexpr int CP = (AX == 0) ? TF + 4 : TF + 3;
  static constexpr int SP = TF + 2;  // slopes per line: faces f0-1 .. f0+TF
  static constexpr int RS = W * CP;  // one staged plane
  static constexpr int SS = W * SP;  // one slope plane
  __host__ __device__ static constexpr int cidx(int line, int pos) { return AX == 0 ? line * CP + pos : pos * W + line; }
  __host__ __device__ static constexpr int sidx(int line, int s) { return AX == 0 ? line * SP + s : s * W + line; }
  // extent of the staged box along x, y, z (the tensor's first three dimensions)
  static constexpr int box(int d) {
    return AX == 0 ? (d == 0 ? CP : (d == 1 ? W : 1)) : (d == 0 ? W : (d == AX ? CP : 1));
  }
};
static_assert((FaceTile<0>::CP * sizeof(double)) % 16 == 0 && (FaceTile<1>::W * sizeof(double)) % 16 == 0,
              "the inner extent of a staged box must be a multiple of 16 bytes");
static_assert(FaceTile<0>::TF % 2 == 0 && FaceTile<1>::W % 2 == 0, "box x origins must be 16-byte aligned");
static_assert((FaceTile<0>::RS * sizeof(double)) % 128 == 0 && (FaceTile<1>::RS * sizeof(double)) % 128 == 0,
              "staged planes keep the 128-byte alignment of the shared-memory base");

// Host-side table of a context's tensor maps: for each state buffer (the two ping-pong states and the
// MUSCL half-step state) and axis, the box of every primitive field and the box of field 0 alone (the
// corrector's time-n alpha_0 plane).
struct FaceMaps {
  const double* buf[3];
  CUtensorMap q[3][3];
  CUtensorMap a0[3][3];
  int ok;  // 1 when every map was built
};

// Encodes the maps of a 2D / 3D mesh of n[0] x n[1] x n[2] cells whose state buffers hold nq primitive
// fields; returns false (and leaves ok = 0) when the layout does not allow a tiled copy or the driver
// entry point is missing.
bool build_face_maps(FaceMaps& m, const double* const bufs[3], int dim, const int n[3], int nq);

// ---------------------------------------------------------------------------------- device side

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for phase `parity` of the barrier, at most `limit` polls (a poll suspends the thread for a
// bounded time); false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// One tiled box copy global -> this CTA's shared memory (no multicast), completing its bytes on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];"
      ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2),
      "r"(c3)
      : "memory");
}

}  // namespace ecg
