// Kapila (PUEq) step kernels: first-order step, MUSCL predictor and MUSCL corrector.
// See ecg_step.cuh for the work decomposition.
#pragma once
#include <cuda_runtime.h>

#include "ecg_kapila_cell.cuh"

namespace ecg {

template <int NP, int DIM, int PASS, int NTM = 0>
struct KapilaStep {
  using FL = Fields<NP, DIM>;
  using TS = TileShape<DIM>;
  static constexpr int H = (PASS == PASS_O1) ? 1 : 2;
  static constexpr int NTH = TS::THREADS;
  static constexpr int NCELL = TS::X * TS::Y * TS::Z;
  static constexpr bool O2 = (PASS != PASS_O1);
  static_assert(NCELL <= NTH, "one thread per cell of the tile");
  static_assert(NTH % 32 == 0 && NTH <= 1024, "whole warps");

  __host__ __device__ static constexpr int ext(int a) { return a == 0 ? TS::X : (a == 1 ? TS::Y : TS::Z); }
  __host__ __device__ static constexpr int lines(int a) { return NCELL / ext(a); }
  __host__ __device__ static constexpr int rlen(int a) { return ext(a) + 2 * H; }
  __host__ __device__ static constexpr int region(int a) { return rlen(a) * lines(a); }
  __host__ __device__ static constexpr int nslope(int a) { return O2 ? (ext(a) + 3) * lines(a) : 0; }
  __host__ __device__ static constexpr int nface(int a) { return (ext(a) + 1) * lines(a); }
  __host__ __device__ static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  __host__ __device__ static constexpr int RMAX() {
    return cmax(region(0), cmax(DIM > 1 ? region(1) : 0, DIM > 2 ? region(2) : 0));
  }
  __host__ __device__ static constexpr int SMAX() {
    return cmax(nslope(0), cmax(DIM > 1 ? nslope(1) : 0, DIM > 2 ? nslope(2) : 0));
  }
  __host__ __device__ static constexpr int FMAX() {
    return cmax(nface(0), cmax(DIM > 1 ? nface(1) : 0, DIM > 2 ? nface(2) : 0));
  }
  static constexpr int NA0 = (PASS == PASS_CORR) ? 1 : 0;  // separate time-n alpha_0 plane
  // passive transports (up to NTM): staged planes, slopes and face fluxes after the others
  static constexpr size_t smem_bytes() {
    return sizeof(double) * ((size_t)RMAX() * (FL::NQ + NA0 + NTM) + (size_t)SMAX() * (FL::NSL + NTM) +
                             (size_t)FMAX() * (FL::NFL + NTM));
  }
};

// Interface detector of CellO2Cartesian::computeLocalSlopes (src/Order2/CellO2Cartesian.cpp:150).
__device__ __forceinline__ bool iface_detect(double aCell, double aOther, double aAfter) {
  return (aCell >= 1.e-4) && (aCell <= 1. - 1.e-4) && ((aOther - aCell) * (aCell - aAfter) >= 1.e-8);
}

template <int NP, int DIM, int PASS, bool PTMU, bool SEED, int TYPES, int NTM = 0>
__global__ void __launch_bounds__(KapilaStep<NP, DIM, PASS, NTM>::NTH,
                                  (PTMU && DIM == 2 && ECG_PTMU_MINB > 0) ? ECG_PTMU_MINB : TileShape<DIM>::MINB)
    k_kapila_step(StepParams P, Geometry G, Model<NP> M0) {
  const Model<NP> M = specialize_eos<NP, TYPES>(M0);
  using K = KapilaStep<NP, DIM, PASS, NTM>;
  using FL = Fields<NP, DIM>;
  using TS = TileShape<DIM>;
  extern __shared__ double smem[];
  constexpr int RS = K::RMAX();
  constexpr int SS = (K::SMAX() > 0) ? K::SMAX() : 1;
  constexpr int FS = K::FMAX();
  double* sq = smem;                                       // [NQ][RS]
  double* sa0 = sq + (size_t)FL::NQ * RS;                  // [NA0][RS]
  double* str = sa0 + (size_t)K::NA0 * RS;                 // [NTM][RS] transports
  double* ssl = str + (size_t)NTM * RS;                    // [NSL + NTM][SS]
  double* sfl = ssl + (K::O2 ? (size_t)(FL::NSL + NTM) * SS : 0);  // [NFL + NTM][FS]
  constexpr int NTA = NTM > 0 ? NTM : 1;

  if (*P.done) return;  // stop condition reached earlier in a captured step sequence
  const int tid = threadIdx.x;
  const int org[3] = {(int)blockIdx.x * TS::X, (int)blockIdx.y * TS::Y, (int)blockIdx.z * TS::Z};
  const int lc[3] = {tid % TS::X, (tid / TS::X) % TS::Y, tid / (TS::X * TS::Y)};
  const int gc[3] = {org[0] + lc[0], org[1] + lc[1], org[2] + lc[2]};
  const bool active = tid < K::NCELL && gc[0] < G.n[0] && gc[1] < G.n[1] && gc[2] < G.n[2];
  const int64_t nn = P.n;
  const int64_t cell = (int64_t)gc[0] + (int64_t)gc[1] * G.n[0] + (int64_t)gc[2] * G.n[0] * G.n[1];

  // time-n state of the own cell: non-conservative terms and U^n
  double an[NP], rn[NP], pn[NP];
  double aa[NP], am[NP], ae[NP], amom[DIM], aE = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    an[k] = rn[k] = pn[k] = 0.;
    aa[k] = am[k] = ae[k] = 0.;
  }
#pragma unroll
  for (int d = 0; d < DIM; d++) amom[d] = 0.;
  if (active) {
    double p0 = P.sn[(int64_t)FL::P * nn + cell];
#pragma unroll
    for (int k = 0; k < NP; k++) {
      an[k] = P.sn[(int64_t)(FL::A + k) * nn + cell];
      rn[k] = P.sn[(int64_t)(FL::R + k) * nn + cell];
      pn[k] = eos_fix_p(M.eos[k], p0);
    }
  }
  // passive transports of the own cell: time-n values and accumulated fluxes
  double tn[NTA], at[NTA];
#pragma unroll
  for (int j = 0; j < NTA; j++) tn[j] = at[j] = 0.;
  if (NTM > 0 && active) {
#pragma unroll
    for (int j = 0; j < NTM; j++)
      if (j < P.ntr) tn[j] = P.sn[(int64_t)(FL::NS + j) * nn + cell];
  }
  double dtmax = 1.e10;
  double wallp[DIM];  // normal momentum flux of the cell's symmetry sides, per axis
#pragma unroll
  for (int d = 0; d < DIM; d++) wallp[d] = 0.;

#pragma unroll
  for (int ax = 0; ax < DIM; ax++) {
    const int T = K::ext(ax), RL = K::rlen(ax), NL = K::lines(ax);
    const int b1 = (ax == 0) ? 1 : 0, b2 = (ax == 2) ? 1 : 2;  // the two other axes
    const int e1 = K::ext(b1);
    const int nax = G.n[ax];
    // ---- stage tile + halo along ax
    for (int e = tid; e < K::region(ax); e += K::NTH) {
      int la = e % RL - K::H, line = e / RL;
      int l1 = line % e1, l2 = line / e1;
      int g[3];
      g[ax] = org[ax] + la;
      g[b1] = org[b1] + l1;
      g[b2] = org[b2] + l2;
      bool in = g[ax] >= 0 && g[ax] < nax && g[b1] < G.n[b1] && g[b2] < G.n[b2];
      if (in) {
        int64_t c = (int64_t)g[0] + (int64_t)g[1] * G.n[0] + (int64_t)g[2] * G.n[0] * G.n[1];
        if (!ECG_IN_BOUNDS(P.stats, c, nn)) continue;
#pragma unroll
        for (int f = 0; f < FL::NQ; f++) sq[f * RS + e] = P.q[(int64_t)f * nn + c];
        if (K::NA0) sa0[e] = P.sn[(int64_t)FL::A * nn + c];
#pragma unroll
        for (int j = 0; j < NTM; j++)
          if (j < P.ntr) str[j * RS + e] = P.q[(int64_t)(FL::NS + j) * nn + c];
      }
    }
    __syncthreads();
    // ---- face slopes (MUSCL): face j between local cells j-1 and j, j in [-1, T+1]
    if (K::O2) {
      for (int e = tid; e < K::nslope(ax); e += K::NTH) {
        int j = e % (T + 3) - 1, line = e / (T + 3);
        int gl = org[ax] + j - 1;
        int rl = line * RL + (j - 1 + K::H), rr = rl + 1;
        if (gl < 0 || gl + 1 >= nax) {
          // a side of the domain: slopes only on a symmetry side, the velocity along the axis over the
          // centre-to-face coordinate (BoundCondWallO2Cartesian::computeSlopes :84-108)
          const int sd = (gl == -1) ? 0 : ((gl == nax - 1) ? 1 : -1);
          if (sd < 0 || G.bc[2 * ax + sd] != ECG_BC_SYMMETRY) continue;
          if (org[b1] + line % e1 >= G.n[b1] || org[b2] + line / e1 >= G.n[b2]) continue;
#pragma unroll
          for (int f = 0; f < FL::NSL + NTM; f++) ssl[f * SS + e] = 0.;
          const double wd = G.wslope[2 * ax + sd];
          if (fabs(wd) > 1.e-8) ssl[(3 * NP + ax) * SS + e] = ddiv(sq[(FL::U + ax) * RS + (sd ? rl : rr)], wd);
          continue;
        }
        double d = G.dcc[ax][gl];
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
#pragma unroll
        for (int j = 0; j < NTM; j++)  // Transport::computeSlopeTransport
          if (j < P.ntr) ssl[(FL::NSL + j) * SS + e] = ddiv(str[j * RS + rr] - str[j * RS + rl], d);
      }
      __syncthreads();
    }
    // ---- face fluxes: face j between local cells j-1 and j, j in [0, T]
    for (int e = tid; e < K::nface(ax); e += K::NTH) {
      int j = e % (T + 1), line = e / (T + 1);
      int l1 = line % e1, l2 = line / e1;
      int gl = org[ax] + j - 1;
      if (gl < 0 || gl + 1 >= nax || org[b1] + l1 >= G.n[b1] || org[b2] + l2 >= G.n[b2]) continue;
      int rl = line * RL + (j - 1 + K::H), rr = rl + 1;
      Thermo<NP> tl, tr;
      double ug[3], vg[3];
      double xl[NTA], xr[NTA];  // transports of the two sides
      if (!K::O2) {
        cell_thermo<NP, DIM>(M, sq, RS, rl, tl, ug);
        cell_thermo<NP, DIM>(M, sq, RS, rr, tr, vg);
#pragma unroll
        for (int t = 0; t < NTM; t++) {
          xl[t] = str[t * RS + rl];
          xr[t] = str[t * RS + rr];
        }
      } else {
        const int fs = line * (T + 3);
        const int f1 = fs + j + 1;                         // this face
        const bool hasL = (gl - 1 >= 0), hasR = (gl + 2 < nax);
        // beyond a symmetry side the opposite slope is the side's and alphaCellAfterOppositeSide is
        // the cell's own time-n alpha (CellO2Cartesian::computeLocalSlopes :68-71); a non-reflecting
        // side has neither
        const bool wL = !hasL && G.bc[2 * ax] == ECG_BC_SYMMETRY;
        const bool wR = !hasR && G.bc[2 * ax + 1] == ECG_BC_SYMMETRY;
        const int f2l = (hasL || wL) ? fs + j : -1;        // face (j-2, j-1)
        const int f2r = (hasR || wR) ? fs + j + 2 : -1;    // face (j, j+1)
        const double* a0 = K::NA0 ? sa0 : sq;              // time-n alpha_0 planes
        double aL = sq[FL::A * RS + rl], aR = sq[FL::A * RS + rr];
        double aLL = hasL ? a0[rl - 1] : (wL ? a0[rl] : 0.), aRR = hasR ? a0[rr + 1] : (wR ? a0[rr] : 0.);
        // THINC is compiled into the generic kernels only (the EOS-specialised ones run without it)
        constexpr bool kThinc = (TYPES == EOS_DYNAMIC);
        constexpr int kLim = code_limiter(TYPES);
        reconstruct_side<NP, DIM, kThinc, kLim>(M, P, sq, RS, rl, ssl, SS, f1, f2l, aL, aR, aLL, G.dfl[ax][gl], 1., tl,
                                                ug);
        reconstruct_side<NP, DIM, kThinc, kLim>(M, P, sq, RS, rr, ssl, SS, f1, f2r, aR, aL, aRR, G.dfr[ax][gl], -1., tr,
                                                vg);
        if (NTM > 0) {  // transports: volume-fraction limiter of each side, Transport::extrapolate
          const int lvL = iface_detect(aL, aR, aLL) ? P.lim[3] : P.lim[2];
          const int lvR = iface_detect(aR, aL, aRR) ? P.lim[3] : P.lim[2];
#pragma unroll
          for (int t = 0; t < NTM; t++) {
            const double s1 = ssl[(FL::NSL + t) * SS + f1];
            const double sl2 = f2l >= 0 ? ssl[(FL::NSL + t) * SS + f2l] : 0.;
            const double sr2 = f2r >= 0 ? ssl[(FL::NSL + t) * SS + f2r] : 0.;
            xl[t] = str[t * RS + rl] + (1. * limiter(lvL, s1, sl2)) * G.dfl[ax][gl];
            xr[t] = str[t * RS + rr] + (-1. * limiter(lvR, s1, sr2)) * G.dfr[ax][gl];
          }
        }
      }
      double ul[3], ur[3], Fn[3];
      to_local(ax, false, ug, ul);
      to_local(ax, false, vg, ur);
      int gf[3];  // the face's left cell, then its right cell: their CFL lengths
      gf[ax] = gl;
      gf[b1] = org[b1] + l1;
      gf[b2] = org[b2] + l2;
      const double lL = cell_lcfl(G, gf[0], gf[1], gf[2]);
      gf[ax] = gl + 1;
      const double lR = cell_lcfl(G, gf[0], gf[1], gf[2]);
      Flux<NP> F;
      hllc<NP>(M, tl, ul, tr, ur, lL, lR, dtmax, Fn, F);
      to_global(ax, false, Fn, F.mom);
#pragma unroll
      for (int k = 0; k < NP; k++) {
        sfl[k * FS + e] = F.a[k];
        sfl[(NP + k) * FS + e] = F.m[k];
        sfl[(2 * NP + k) * FS + e] = F.en[k];
      }
#pragma unroll
      for (int d = 0; d < DIM; d++) sfl[(3 * NP + d) * FS + e] = F.mom[d];
      sfl[(3 * NP + DIM) * FS + e] = F.E;
      sfl[(3 * NP + DIM + 1) * FS + e] = F.sM;
      sfl[(3 * NP + DIM + 2) * FS + e] = F.uStar;
#pragma unroll
      for (int t = 0; t < NTM; t++)  // Transport::solveRiemann: upwind by sM
        sfl[(FL::NFL + t) * FS + e] = (F.sM > 0.) ? xl[t] * F.sM : xr[t] * F.sM;
    }
    __syncthreads();
    // ---- accumulate the two faces of this axis into the own cell (left +, right -)
    if (active) {
      int la = lc[ax];
      int line = lc[b1] + lc[b2] * e1;
      const double cA = cell_coefA(G, ax, gc[0], gc[1], gc[2]);
#pragma unroll
      for (int side = 0; side < 2; side++) {
        int j = la + side;
        int gl = org[ax] + j - 1;
        if (gl < 0 || gl + 1 >= nax) continue;  // boundary face: handled below
        int e = line * (T + 1) + j;
        if (!ECG_IN_BOUNDS(P.stats, e, FS)) continue;
        Flux<NP> F;
#pragma unroll
        for (int k = 0; k < NP; k++) {
          F.a[k] = sfl[k * FS + e];
          F.m[k] = sfl[(NP + k) * FS + e];
          F.en[k] = sfl[(2 * NP + k) * FS + e];
        }
#pragma unroll
        for (int d = 0; d < DIM; d++) F.mom[d] = sfl[(3 * NP + d) * FS + e];
        F.E = sfl[(3 * NP + DIM) * FS + e];
        F.sM = sfl[(3 * NP + DIM + 1) * FS + e];
        F.uStar = sfl[(3 * NP + DIM + 2) * FS + e];
        acc_face<NP, DIM>(cA, side == 0, F, an, pn, aa, am, ae, amom, aE);
#pragma unroll
        for (int t = 0; t < NTM; t++) {  // Transport::addFlux / addNonCons (time-n value), or subtract
          if (t >= P.ntr) continue;
          const double ft = sfl[(FL::NFL + t) * FS + e];
          if (side == 0) {
            at[t] += cA * ft;
            at[t] += -cA * tn[t] * F.sM;
          } else {
            at[t] -= cA * ft;
            at[t] -= -cA * tn[t] * F.sM;
          }
        }
      }
      // a symmetry side of this cell along ax: its flux is computed now, while the slopes of this axis
      // are staged, and subtracted with the other boundary faces below (reference face order)
      const int sd = (gc[ax] == 0) ? 0 : ((gc[ax] == nax - 1) ? 1 : -1);
      if (sd >= 0 && G.bc[2 * ax + sd] == ECG_BC_SYMMETRY) {
        const int rc = line * RL + la + K::H;
        Thermo<NP> t;
        double ug[3], ul[3];
        if (K::O2) {
          const int fs = line * (T + 3);
          wall_side<NP, DIM>(M, P.lim, sq, RS, rc, ssl, SS, fs + la + 1 + sd, fs + la + 2 - sd, an[0],
                             G.wdist[2 * ax + sd], t, ug);
        } else {
          cell_thermo<NP, DIM>(M, sq, RS, rc, t, ug);
        }
        to_local(ax, sd == 0, ug, ul);
        wallp[ax] = wall_pstar<NP>(t, ul, cell_lcfl(G, gc[0], gc[1], gc[2]), dtmax);
      }
    }
    __syncthreads();
  }

  // per-thread counters, reduced per block at the end
  CellCounters cc;
  CellPrim<NP, DIM> cp;
  if (active) {
    // ---- boundary faces (non-reflecting: HLLC(cell, cell), BoundCondNonReflecting::solveRiemannBoundary
    //      src/BoundConds/BoundCondNonReflecting.cpp:62; symmetry: the flux computed in the axis pass),
    //      subtracted from the cell (BoundCond::computeFlux :61)
#pragma unroll
    for (int bf = 0; bf < 2 * DIM; bf++) {
      int ax = bf >> 1;
      bool neg = (bf & 1) == 0;
      if (neg ? (gc[ax] != 0) : (gc[ax] != G.n[ax] - 1)) continue;
      double sMb = 0.;
      const double cAb = cell_coefA(G, ax, gc[0], gc[1], gc[2]);
      if (G.bc[bf] == ECG_BC_SYMMETRY)
        wall_acc<NP, DIM>(ax, neg, wallp[ax], cAb, an, pn, aa, am, ae, amom, aE);
      else
        boundary_face<NP, DIM>(M, P.q, nn, cell, ax, neg, cell_lcfl(G, gc[0], gc[1], gc[2]), cAb, dtmax, an, pn, aa,
                               am, ae, amom, aE, &sMb);
#pragma unroll
      for (int t = 0; t < NTM; t++) {  // transports: T sM on a non-reflecting side, nothing on a symmetry side
        if (t >= P.ntr) continue;
        const double ft = (G.bc[bf] == ECG_BC_SYMMETRY) ? 0. : P.q[(int64_t)(FL::NS + t) * nn + cell] * sMb;
        at[t] -= cAb * ft;
        at[t] -= -cAb * tn[t] * sMb;
      }
    }

    kapila_rebuild<NP, DIM, PASS>(P, M, nn, cell, *P.dt, an, rn, pn, aa, am, ae, amom, aE, cp);
    if (NTM > 0) {  // Cell::timeEvolution :294-298 / CellO2::predictionOrdre2 :121-125
      const double scale = (PASS == PASS_PRED) ? 0.5 * *P.dt : *P.dt;
#pragma unroll
      for (int t = 0; t < NTM; t++)
        if (t < P.ntr) P.out[(int64_t)(FL::NS + t) * nn + cell] = tn[t] + at[t] * scale;
    }
  }
  // learned seed of the pressure relaxation, gated on the plain start (all lanes of the warp)
  SeedGate<NP> sg;
  if (SEED && !PTMU) seed_gate<NP, DIM>(P, M, active, cp, sg);
  if (SEED && PTMU) ptmu_seed_gate<NP, DIM>(P, M, active, cp, sg, cc);
  if (active) kapila_finish<NP, DIM, PASS, PTMU, SEED, (TYPES == EOS_DYNAMIC)>(P, M, nn, cell, cp, sg, cc);
  block_counters(P.stats, cc.relax, cc.iters, cc.fallback, cc.seeded, cc.rejected, cc.nonfinite, cc.ptmu, cc.iters, true);
  if (PTMU)
    block_ptmu_counters(P.stats, cc.pc.solve, cc.pc.outer, cc.pc.tsat_calls, cc.pc.tsat_iters, cc.pc.tsat_max,
                        cc.pc.seeded, cc.pc.rejected);

  // ---- dtMax: block min, one atomic per block
  __shared__ double red[32];
  double v = dtmax;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((tid & 31) == 0) red[tid >> 5] = v;
  __syncthreads();
  if (tid < 32) {
    v = (tid < K::NTH / 32) ? red[tid] : 1.e10;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (tid == 0) atomic_min_pos_double(P.dtmax_bits, v);
  }
}

}  // namespace ecg

