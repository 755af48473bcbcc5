// Split form of a Kapila step pass for 2D and 3D meshes: one face-flux kernel per axis, then one cell
// kernel.
//
// The fused pass (ecg_kapila_kernel.cuh) stages a tile per axis, computes its faces and accumulates
// them in one kernel: every block runs the whole pass (both axes' slopes, reconstructions and HLLC
// solves, then the relaxation) with a barrier after each phase, so warps whose faces took the cheap
// HLLC branch wait at the barrier for the ones sampling a star state, and the kernel's code (one copy
// of the face work per axis) is larger than the instruction cache.  The split form trades HBM
// traffic, of which the pass uses a few percent, for latency:
//   k_kapila_faces<AX>  one thread per face normal to axis AX: stage the cells and the face slopes of a
//                        block (one barrier), then reconstruct both sides and solve HLLC exactly as the
//                        fused pass does, including the domain sides (non-reflecting: HLLC(cell, cell) in
//                        the side's frame; symmetry: the reflecting flux of the MUSCL buffer cell), and
//                        store the face flux (3N + d + 3 doubles) in a face array of the axis;
//                        min-reduce lCFL/|s| into dtMax;
//   k_kapila_cells       one thread per cell, no shared memory and no barrier but the counters': add
//                        and subtract the stored fluxes in the reference's face order (X faces, Y faces,
//                        Z faces, then sides Xm, Xp, Ym, Yp, Zm, Zp, src/Meshes/MeshCartesian.cpp:281-557)
//                        with the same non-conservative terms, then buildPrim, relaxations, energy
//                        correction and store (kapila_rebuild / kapila_finish).
// Every flux is computed once, by the same device functions in the same operation order, and each cell
// accumulates the same values in the same order, so the split and fused forms give identical bits.
//
// Face arrays (per axis, structure of arrays, NFL components of nfaces(AX) doubles): the face between
// cells f-1 and f along AX (f = 0 and f = n_AX are the domain sides) of the line at the other
// coordinates has index  f + (nx+1)(j + ny k)  (X),  i + nx (f + (ny+1) k)  (Y),  i + nx (j + ny f)  (Z),
// so that consecutive threads of either kernel touch consecutive faces.
#pragma once
#include "ecg_kapila_kernel.cuh"
#include "ecg_tma.cuh"

namespace ecg {

__device__ __forceinline__ int64_t split_fid(const int n[3], int ax, int f, int i, int j, int k) {
  if (ax == 0) return (int64_t)f + (int64_t)(n[0] + 1) * ((int64_t)j + (int64_t)n[1] * k);
  if (ax == 1) return (int64_t)i + (int64_t)n[0] * ((int64_t)f + (int64_t)(n[1] + 1) * k);
  return (int64_t)i + (int64_t)n[0] * ((int64_t)j + (int64_t)n[1] * f);
}

template <int NP, int DIM, int AX, int PASS>
struct FaceKernelShape {
  using FL = Fields<NP, DIM>;
  using FT = FaceTile<AX>;
  static constexpr bool O2 = (PASS != PASS_O1);
  static constexpr int NA0 = (PASS == PASS_CORR) ? 1 : 0;  // separate time-n alpha_0 plane
  static constexpr size_t staged_bytes() { return sizeof(double) * (size_t)FT::RS * (FL::NQ + NA0); }
  // staged planes, slope planes, the staging mbarrier, and room to align the base to 128 bytes
  static constexpr size_t smem_bytes() {
    return staged_bytes() + (O2 ? sizeof(double) * (size_t)FT::SS * FL::NSL : 0) + sizeof(uint64_t) + 128;
  }
};

// Resident blocks per SM asked of the face and cell kernels (registers 65536 / (128 x MINB)).  Measured
// on one B200 with the branch-free division (per-kernel CUDA events, 100 steps): 3D three-phase cavity
// 256^3: face kernels at 6 blocks (80 registers) 2.35 / 2.11 ms (X / Y faces), at 5 2.43 / 2.13 ms;
// cell kernel at 6 blocks 2.96 ms, at 5 (96 registers, fewer spills) 2.90 ms; 2D shock-bubble 2048^2:
// face kernels at 8 blocks 0.353 / 0.328 ms, at 7 0.354 / 0.322 ms; cell kernel at 6 0.393 ms, at 5
// 0.390 ms.
#ifndef ECG_FACE_MINB_2D
#define ECG_FACE_MINB_2D 7
#endif
#ifndef ECG_FACE_MINB_3D
#define ECG_FACE_MINB_3D 6
#endif
#ifndef ECG_CELL_MINB
#define ECG_CELL_MINB 5
#endif
// The cell kernels with the learned pressure seed: the network's MMA fragments and features need
// registers (at 96 the seeded kernels spilled about 600 B).  Measured (seeded arm, CUDA events, 100
// steps): 3D cavity 256^3 at 5 blocks per SM 684.8 M cell-updates/s, at 4 (128 registers) 708.8 M, at 3
// 681.9 M; 2D shock-bubble 2048^2 1668.8 M, 1851.1 M and 1700.3 M.
#ifndef ECG_CELL_SEED_MINB
#define ECG_CELL_SEED_MINB 4
#endif
// The p-T-mu cell kernels run one warp per block: their cells take very different numbers of Newton
// iterations, and in 4-warp blocks the warps that finish first waited at the block's counter reduction
// for the slowest one (barrier stalls were 5.6 of 12.4 cycles between issues on the 1024^2 expansion),
// holding their slots; a one-warp block frees its slot for the next block as soon as it is done.
// 16 such blocks per SM keep the 128-register budget of 4 blocks of 4 warps.
#ifndef ECG_CELL_PTMU_THREADS
#define ECG_CELL_PTMU_THREADS 32
#endif
#ifndef ECG_CELL_PTMU_MINB
#define ECG_CELL_PTMU_MINB (512 / ECG_CELL_PTMU_THREADS)
#endif
constexpr int CELL_THREADS = 128;
__host__ __device__ constexpr int cell_threads(bool ptmu) { return ptmu ? ECG_CELL_PTMU_THREADS : CELL_THREADS; }

template <int NP, int DIM, int AX, int PASS, int TYPES>
__global__ void __launch_bounds__(FaceTile<AX>::NTH, DIM == 2 ? ECG_FACE_MINB_2D : ECG_FACE_MINB_3D)
    k_kapila_faces(StepParams P, Geometry G, Model<NP> M0, double* __restrict__ flux,
                   const __grid_constant__ CUtensorMap mq, const __grid_constant__ CUtensorMap ma0, int tma) {
  const Model<NP> M = specialize_eos<NP, TYPES>(M0);
  using FT = FaceTile<AX>;
  using KS = FaceKernelShape<NP, DIM, AX, PASS>;
  using FL = Fields<NP, DIM>;
  constexpr bool O2 = KS::O2;
  constexpr int RS = FT::RS, SS = FT::SS, CP = FT::CP;
  extern __shared__ unsigned char smem_raw[];
  double* smem = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  double* sq = smem;                                // [NQ][RS]
  double* sa0 = sq + (size_t)FL::NQ * RS;           // [NA0][RS]
  double* ssl = sa0 + (size_t)KS::NA0 * RS;         // [NSL][SS]
  const double* a0 = KS::NA0 ? sa0 : sq;            // time-n alpha_0 plane

  if (*P.done) return;
  const int tid = threadIdx.x;
  const int nax = G.n[AX];
  const int ob = (AX == 0) ? 1 : 0;                 // the lines' axis
  const int f0 = (int)(AX == 0 ? blockIdx.x : blockIdx.y) * FT::TF;
  const int l0 = (int)(AX == 0 ? blockIdx.y : blockIdx.x) * FT::W;
  const int third = (int)blockIdx.z;                // Z for X and Y faces, Y for Z faces
  const int64_t nn = P.n;
  // global cell coordinates of (line, position along AX)
  auto coords = [&](int line, int gpos, int g[3]) {
    g[AX] = gpos;
    g[ob] = l0 + line;
    g[AX == 2 ? 1 : 2] = third;
  };

  // ---- stage the cells f0-2 .. f0-3+CP of every line
  if (tma) {
    // one tensor copy of the box (x, y[, z], field) for all primitive fields, one for the time-n
    // alpha_0 plane; cells outside the mesh arrive as zeros
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + KS::staged_bytes() / sizeof(double) +
                                                (O2 ? (size_t)FT::SS * FL::NSL : 0));
    if (tid == 0) mbar_init(bar, 1);
    __syncthreads();
    if (tid == 0) {
      mbar_expect_tx(bar, (uint32_t)KS::staged_bytes());
      int o[3];  // box origin along x, y, z
      o[AX] = f0 - 2;
      o[ob] = l0;
      o[AX == 2 ? 1 : 2] = third;
      if (DIM == 3) {
        tma_load_4d(sq, &mq, bar, o[0], o[1], o[2], 0);
        if (KS::NA0) tma_load_4d(sa0, &ma0, bar, o[0], o[1], o[2], FL::A);
      } else {
        tma_load_3d(sq, &mq, bar, o[0], o[1], 0);
        if (KS::NA0) tma_load_3d(sa0, &ma0, bar, o[0], o[1], FL::A);
      }
    }
    // bounded wait; a copy that never lands is reported to the host (the step then fails)
    if (!mbar_wait_bounded(bar, 0, 1 << 22) && (tid & 31) == 0) atomicAdd(&P.stats->staging_timeouts, 1ull);
  } else {
    for (int e = tid; e < RS; e += FT::NTH) {
      const int line = AX == 0 ? e / CP : e % FT::W, pos = AX == 0 ? e % CP : e / FT::W;
      int g[3];
      coords(line, f0 - 2 + pos, g);
      if (g[AX] >= 0 && g[AX] < nax && g[ob] < G.n[ob]) {
        const int64_t c = (int64_t)g[0] + (int64_t)g[1] * G.n[0] + (int64_t)g[2] * G.n[0] * G.n[1];
        if (!ECG_IN_BOUNDS(P.stats, c, nn)) continue;
#pragma unroll
        for (int f = 0; f < FL::NQ; f++) sq[f * RS + e] = P.q[(int64_t)f * nn + c];
        if (KS::NA0) sa0[e] = P.sn[(int64_t)FL::A * nn + c];
      }
    }
  }
  __syncthreads();
  // ---- face slopes (MUSCL): slope s at face g = f0 - 1 + s, between cells g-1 and g
  if (O2) {
    for (int e = tid; e < SS; e += FT::NTH) {
      const int line = AX == 0 ? e / FT::SP : e % FT::W, s = AX == 0 ? e % FT::SP : e / FT::W;
      const int gl = f0 - 2 + s;  // left cell of the face
      if (l0 + line >= G.n[ob]) continue;
      const int rl = FT::cidx(line, s), rr = FT::cidx(line, s + 1);
      if (gl < 0 || gl + 1 >= nax) {
        // a side of the domain: slopes only on a symmetry side, the velocity along the axis over the
        // centre-to-face coordinate (BoundCondWallO2Cartesian::computeSlopes :84-108)
        const int sd = (gl == -1) ? 0 : ((gl == nax - 1) ? 1 : -1);
        if (sd < 0 || G.bc[2 * AX + sd] != ECG_BC_SYMMETRY) continue;
#pragma unroll
        for (int f = 0; f < FL::NSL; f++) ssl[f * SS + e] = 0.;
        const double wd = G.wslope[2 * AX + sd];
        if (fabs(wd) > 1.e-8) ssl[(3 * NP + AX) * SS + e] = ddiv(sq[(FL::U + AX) * RS + (sd ? rl : rr)], wd);
        continue;
      }
      const double d = G.dcc[AX][gl];
#pragma unroll
      for (int k = 0; k < NP; k++) {
        ssl[k * SS + e] = ddiv(sq[(FL::A + k) * RS + rr] - sq[(FL::A + k) * RS + rl], d);
        ssl[(NP + k) * SS + e] = ddiv(sq[(FL::R + k) * RS + rr] - sq[(FL::R + k) * RS + rl], d);
        double pr = eos_fix_p(M.eos[k], sq[FL::P * RS + rr]), pl = eos_fix_p(M.eos[k], sq[FL::P * RS + rl]);
        ssl[(2 * NP + k) * SS + e] = ddiv(pr - pl, d);
      }
#pragma unroll
      for (int dd = 0; dd < DIM; dd++)
        ssl[(3 * NP + dd) * SS + e] = ddiv(sq[(FL::U + dd) * RS + rr] - sq[(FL::U + dd) * RS + rl], d);
    }
    __syncthreads();
  }

  // ---- one face per thread
  double dtmax = 1.e10;
  {
    const int line = AX == 0 ? tid / FT::TF : tid % FT::W, fl = AX == 0 ? tid % FT::TF : tid / FT::W;
    const int f = f0 + fl;
    int g[3];
    coords(line, f, g);
    // (bounds-checked builds: the staged cells this face reads, positions fl .. fl + 3 of its line)
    if (f <= nax && g[ob] < G.n[ob] && ECG_IN_BOUNDS(P.stats, FT::cidx(line, fl), RS) &&
        ECG_IN_BOUNDS(P.stats, FT::cidx(line, fl + 3), RS)) {
      Flux<NP> F;
      double Fn[3];
      const int gl = f - 1;
      if (f == 0 || f == nax) {
        // a side: non-reflecting HLLC(cell, cell) in the side's frame (BoundCondNonReflecting::
        // solveRiemannBoundary src/BoundConds/BoundCondNonReflecting.cpp:62), or a symmetry side's
        // reflecting flux (ModUEq::solveRiemannWall src/Models/UEq/ModUEq.cpp:452) of the buffer cell,
        // MUSCL-extrapolated towards the side (BoundCondWallO2Cartesian::solveRiemann :111-141)
        const int sd = (f == 0) ? 0 : 1;
        const bool neg = sd == 0;
        const int rc = FT::cidx(line, sd == 0 ? fl + 2 : fl + 1);
        int gc[3] = {g[0], g[1], g[2]};  // the side's cell
        gc[AX] = sd == 0 ? 0 : nax - 1;
        const double lc = cell_lcfl(G, gc[0], gc[1], gc[2]);
        Thermo<NP> t;
        double ug[3], ul[3];
        if (G.bc[2 * AX + sd] == ECG_BC_SYMMETRY) {
          if (O2) {
            const int fw = FT::sidx(line, fl + 1), fo = FT::sidx(line, sd == 0 ? fl + 2 : fl);
            wall_side<NP, DIM>(M, P.lim, sq, RS, rc, ssl, SS, fw, fo, a0[rc], G.wdist[2 * AX + sd], t, ug);
          } else {
            cell_thermo<NP, DIM>(M, sq, RS, rc, t, ug);
          }
          to_local(AX, neg, ug, ul);
          const double pstar = wall_pstar<NP>(t, ul, lc, dtmax);
#pragma unroll
          for (int k = 0; k < NP; k++) F.a[k] = F.m[k] = F.en[k] = 0.;
          F.E = 0.;
          F.sM = 0.;
          F.uStar = 0.;
          Fn[0] = pstar;
          Fn[1] = 0.;
          Fn[2] = 0.;
        } else {
          cell_thermo<NP, DIM>(M, sq, RS, rc, t, ug);
          to_local(AX, neg, ug, ul);
          hllc<NP>(M, t, ul, t, ul, lc, lc, dtmax, Fn, F);
        }
        to_global(AX, neg, Fn, F.mom);
      } else {
        // internal face between cells gl and gl + 1 (positions fl + 1 and fl + 2)
        const int rl = FT::cidx(line, fl + 1), rr = FT::cidx(line, fl + 2);
        Thermo<NP> tl, tr;
        double ug[3], vg[3];
        if (!O2) {
          cell_thermo<NP, DIM>(M, sq, RS, rl, tl, ug);
          cell_thermo<NP, DIM>(M, sq, RS, rr, tr, vg);
        } else {
          const int f1 = FT::sidx(line, fl + 1);  // this face
          const bool hasL = (gl - 1 >= 0), hasR = (gl + 2 < nax);
          // beyond a symmetry side the opposite slope is the side's and alphaCellAfterOppositeSide is the
          // cell's own time-n alpha (CellO2Cartesian::computeLocalSlopes :68-71); a non-reflecting side
          // has neither
          const bool wL = !hasL && G.bc[2 * AX] == ECG_BC_SYMMETRY;
          const bool wR = !hasR && G.bc[2 * AX + 1] == ECG_BC_SYMMETRY;
          const int f2l = (hasL || wL) ? FT::sidx(line, fl) : -1;      // face (gl-1, gl)
          const int f2r = (hasR || wR) ? FT::sidx(line, fl + 2) : -1;  // face (gl+1, gl+2)
          const double aL = sq[FL::A * RS + rl], aR = sq[FL::A * RS + rr];
          const double aLL = hasL ? a0[FT::cidx(line, fl)] : (wL ? a0[rl] : 0.);
          const double aRR = hasR ? a0[FT::cidx(line, fl + 3)] : (wR ? a0[rr] : 0.);
          constexpr bool kThinc = (TYPES == EOS_DYNAMIC);
          constexpr int kLim = code_limiter(TYPES);
          reconstruct_side<NP, DIM, kThinc, kLim>(M, P, sq, RS, rl, ssl, SS, f1, f2l, aL, aR, aLL, G.dfl[AX][gl], 1.,
                                                  tl, ug);
          reconstruct_side<NP, DIM, kThinc, kLim>(M, P, sq, RS, rr, ssl, SS, f1, f2r, aR, aL, aRR, G.dfr[AX][gl], -1.,
                                                  tr, vg);
        }
        double ul[3], ur[3];
        to_local(AX, false, ug, ul);
        to_local(AX, false, vg, ur);
        int gf[3] = {g[0], g[1], g[2]};  // the face's left cell, then its right cell: their CFL lengths
        gf[AX] = gl;
        const double lL = cell_lcfl(G, gf[0], gf[1], gf[2]);
        gf[AX] = gl + 1;
        const double lR = cell_lcfl(G, gf[0], gf[1], gf[2]);
        hllc<NP>(M, tl, ul, tr, ur, lL, lR, dtmax, Fn, F);
        to_global(AX, false, Fn, F.mom);
      }
      const int64_t nfa = split_nfaces(G.n, AX);
      const int64_t fid = split_fid(G.n, AX, f, g[0], g[1], g[2]);
      if (ECG_IN_BOUNDS(P.stats, fid, nfa)) {
        double* out = flux + fid;
#pragma unroll
        for (int k = 0; k < NP; k++) {
          out[(int64_t)k * nfa] = F.a[k];
          out[(int64_t)(NP + k) * nfa] = F.m[k];
          out[(int64_t)(2 * NP + k) * nfa] = F.en[k];
        }
#pragma unroll
        for (int d = 0; d < DIM; d++) out[(int64_t)(3 * NP + d) * nfa] = F.mom[d];
        out[(int64_t)(3 * NP + DIM) * nfa] = F.E;
        out[(int64_t)(3 * NP + DIM + 1) * nfa] = F.sM;
        out[(int64_t)(3 * NP + DIM + 2) * nfa] = F.uStar;
      }
    }
  }

  // ---- dtMax: block min, one atomic per block
  __shared__ double red[32];
  double v = dtmax;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((tid & 31) == 0) red[tid >> 5] = v;
  __syncthreads();
  if (tid < 32) {
    v = (tid < FT::NTH / 32) ? red[tid] : 1.e10;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (tid == 0) atomic_min_pos_double(P.dtmax_bits, v);
  }
}

template <int NP, int DIM>
__device__ __forceinline__ void load_face_flux(const double* __restrict__ fl, int64_t nfa, int64_t fid, Flux<NP>& F,
                                               DevStats* st) {
  if (!ECG_IN_BOUNDS(st, fid, nfa)) fid = 0;
  const double* p = fl + fid;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    F.a[k] = p[(int64_t)k * nfa];
    F.m[k] = p[(int64_t)(NP + k) * nfa];
    F.en[k] = p[(int64_t)(2 * NP + k) * nfa];
  }
#pragma unroll
  for (int d = 0; d < DIM; d++) F.mom[d] = p[(int64_t)(3 * NP + d) * nfa];
  F.E = p[(int64_t)(3 * NP + DIM) * nfa];
  F.sM = p[(int64_t)(3 * NP + DIM + 1) * nfa];
  F.uStar = p[(int64_t)(3 * NP + DIM + 2) * nfa];
}

template <int NP, int DIM, int PASS, bool PTMU, bool SEED, int TYPES>
__global__ void __launch_bounds__(cell_threads(PTMU),
                                  PTMU ? ECG_CELL_PTMU_MINB : (SEED ? ECG_CELL_SEED_MINB : ECG_CELL_MINB))
    k_kapila_cells(StepParams P, Geometry G, Model<NP> M0, const double* __restrict__ fx,
                   const double* __restrict__ fy, const double* __restrict__ fz) {
  const Model<NP> M = specialize_eos<NP, TYPES>(M0);
  using FL = Fields<NP, DIM>;
  if (*P.done) return;
  const int64_t nn = P.n;
  const int64_t cell = (int64_t)blockIdx.x * cell_threads(PTMU) + threadIdx.x;
  const bool active = cell < nn;
  int g[3] = {0, 0, 0};
  if (active) {
    g[0] = (int)(cell % G.n[0]);
    g[1] = (int)((cell / G.n[0]) % G.n[1]);
    g[2] = (int)(cell / ((int64_t)G.n[0] * G.n[1]));
  }
  double an[NP], rn[NP], pn[NP];
  double aa[NP], am[NP], ae[NP], amom[DIM], aE = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    an[k] = rn[k] = pn[k] = 0.;
    aa[k] = am[k] = ae[k] = 0.;
  }
#pragma unroll
  for (int d = 0; d < DIM; d++) amom[d] = 0.;
  CellCounters cc;
  CellPrim<NP, DIM> cp;
  if (active) {
    const double p0 = P.sn[(int64_t)FL::P * nn + cell];
#pragma unroll
    for (int k = 0; k < NP; k++) {
      an[k] = P.sn[(int64_t)(FL::A + k) * nn + cell];
      rn[k] = P.sn[(int64_t)(FL::R + k) * nn + cell];
      pn[k] = eos_fix_p(M.eos[k], p0);
    }
    const double* fa[3] = {fx, fy, fz};
    // internal faces, axis by axis: the left face added, the right face subtracted
#pragma unroll
    for (int ax = 0; ax < DIM; ax++) {
      const int64_t nfa = split_nfaces(G.n, ax);
      const double cA = cell_coefA(G, ax, g[0], g[1], g[2]);
      Flux<NP> F;
      if (g[ax] >= 1) {
        load_face_flux<NP, DIM>(fa[ax], nfa, split_fid(G.n, ax, g[ax], g[0], g[1], g[2]), F, P.stats);
        acc_face<NP, DIM>(cA, true, F, an, pn, aa, am, ae, amom, aE);
      }
      if (g[ax] + 1 <= G.n[ax] - 1) {
        load_face_flux<NP, DIM>(fa[ax], nfa, split_fid(G.n, ax, g[ax] + 1, g[0], g[1], g[2]), F, P.stats);
        acc_face<NP, DIM>(cA, false, F, an, pn, aa, am, ae, amom, aE);
      }
    }
    // the domain sides Xm, Xp, Ym, Yp, Zm, Zp, subtracted from the cell (BoundCond::computeFlux
    // src/BoundConds/BoundCond.cpp:61)
#pragma unroll
    for (int bf = 0; bf < 2 * DIM; bf++) {
      const int ax = bf >> 1;
      const bool neg = (bf & 1) == 0;
      if (neg ? (g[ax] != 0) : (g[ax] != G.n[ax] - 1)) continue;
      Flux<NP> F;
      load_face_flux<NP, DIM>(fa[ax], split_nfaces(G.n, ax), split_fid(G.n, ax, neg ? 0 : G.n[ax], g[0], g[1], g[2]),
                              F, P.stats);
      acc_face<NP, DIM>(cell_coefA(G, ax, g[0], g[1], g[2]), false, F, an, pn, aa, am, ae, amom, aE);
    }
    kapila_rebuild<NP, DIM, PASS>(P, M, nn, cell, *P.dt, an, rn, pn, aa, am, ae, amom, aE, cp);
  }
  SeedGate<NP> sg;
  if (SEED && !PTMU) seed_gate<NP, DIM>(P, M, active, cp, sg);
  if (SEED && PTMU) ptmu_seed_gate<NP, DIM>(P, M, active, cp, sg, cc);
  if (active) kapila_finish<NP, DIM, PASS, PTMU, SEED, (TYPES == EOS_DYNAMIC)>(P, M, nn, cell, cp, sg, cc);
  block_counters(P.stats, cc.relax, cc.iters, cc.fallback, cc.seeded, cc.rejected, cc.nonfinite, cc.ptmu, cc.iters, true);
  if (PTMU)
    block_ptmu_counters(P.stats, cc.pc.solve, cc.pc.outer, cc.pc.tsat_calls, cc.pc.tsat_iters, cc.pc.tsat_max,
                        cc.pc.seeded, cc.pc.rejected);
}

template <int NP, int DIM, int AX, int PASS, int TYPES>
cudaError_t launch_faces(const StepParams& P, const Geometry& G, const Model<NP>& M, cudaStream_t s, bool prepare) {
  using FT = FaceTile<AX>;
  auto kern = k_kapila_faces<NP, DIM, AX, PASS, TYPES>;
  const size_t sm = FaceKernelShape<NP, DIM, AX, PASS>::smem_bytes();
  if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  // tensor maps of the buffers this pass reads (TMA staging), when the context built them
  CUtensorMap mq{}, ma0{};
  int tma = 0;
  if (P.fmaps && P.fmaps->ok) {
    const CUtensorMap *q = nullptr, *a = nullptr;
    for (int b = 0; b < 3; b++) {
      if (P.fmaps->buf[b] && P.fmaps->buf[b] == P.q) q = &P.fmaps->q[b][AX];
      if (P.fmaps->buf[b] && P.fmaps->buf[b] == P.sn) a = &P.fmaps->a0[b][AX];
    }
    if (q && (PASS != PASS_CORR || a)) {
      mq = *q;
      if (a) ma0 = *a;
      tma = 1;
    }
  }
  const int nax = G.n[AX], ob = AX == 0 ? 1 : 0, third = AX == 2 ? G.n[1] : G.n[2];
  dim3 grid, blk(FT::NTH);
  const unsigned gf = (unsigned)((nax + 1 + FT::TF - 1) / FT::TF), gl = (unsigned)((G.n[ob] + FT::W - 1) / FT::W);
  if (AX == 0) grid = dim3(gf, gl, (unsigned)third);
  else grid = dim3(gl, gf, (unsigned)third);
  kern<<<grid, blk, sm, s>>>(P, G, M, P.flux[AX], mq, ma0, tma);
  return cudaGetLastError();
}

// One pass in split form: the face kernels of every axis, then the cell kernel.  With prepare, only
// the kernels' attributes are set.
template <int NP, int DIM, int PASS, bool PTMU, bool SEED, int TYPES>
cudaError_t launch_split(const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps, cudaStream_t s,
                         bool prepare) {
  Model<NP> M;
  for (int k = 0; k < NP; k++) M.eos[k] = make_eos_params(eos[k]);
  M.eps = eps;
  cudaError_t e = launch_faces<NP, DIM, 0, PASS, TYPES>(P, G, M, s, prepare);
  if (e == cudaSuccess && P.split_ev && !prepare) e = cudaEventRecord(P.split_ev[0], s);
  if (e == cudaSuccess) e = launch_faces<NP, DIM, 1, PASS, TYPES>(P, G, M, s, prepare);
  if (e == cudaSuccess && P.split_ev && !prepare) e = cudaEventRecord(P.split_ev[1], s);
  if (DIM > 2 && e == cudaSuccess) e = launch_faces<NP, DIM, (DIM > 2 ? 2 : 0), PASS, TYPES>(P, G, M, s, prepare);
  if (DIM > 2 && e == cudaSuccess && P.split_ev && !prepare) e = cudaEventRecord(P.split_ev[2], s);
  if (e != cudaSuccess || prepare) return e;
  constexpr int CT = cell_threads(PTMU);
  const unsigned blocks = (unsigned)((P.n + CT - 1) / CT);
  k_kapila_cells<NP, DIM, PASS, PTMU, SEED, TYPES><<<blocks, CT, 0, s>>>(P, G, M, P.flux[0], P.flux[1],
                                                                                 DIM > 2 ? P.flux[2] : nullptr);
  return cudaGetLastError();
}

}  // namespace ecg
