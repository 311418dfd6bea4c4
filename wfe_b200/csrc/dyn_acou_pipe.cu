// Persistent, pipelined vertically implicit w - pi' column kernel
// (src/dynamics/kernels.cu:545-645, the reference's k_acou_wpi).
//
// The column kernels that load their inputs with ordinary loads wait on
// memory: a CTA issues its loads, then every level lane waits at the barrier
// in front of the serial Thomas sweep, and with two CTAs per SM little else
// is resident to keep loads in flight.  Here a CTA is persistent and owns a
// strided list of tiles (CX columns of one row, all levels).  One producer
// warp streams each tile's input boxes into a ring of NST shared-memory
// stages with bulk tensor loads (cp.async.bulk.tensor, no multicast: the
// maps cover this GPU's own fields only), signalling a "full" mbarrier per
// stage with the transaction bytes; the consumer warps take the tiles in
// order: phases 1-3 from shared memory into registers and the row arrays,
// release the stage (its "empty" mbarrier) so the next tile's loads start
// while this tile is still being solved, the Thomas sweep in the first CX
// threads, then phase 5 from registers and the solution.  Every wait on a
// barrier is bounded: on a timeout the kernel sets *err and leaves.
//
// The arithmetic is the chunked column kernel's (dyn_acou.cu), expression by
// expression and in the same order, so the results are bit-identical to it.
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "acou_pcr.cuh"
#include "core.cuh"
#include "kernels.cuh"
#include "dyn_common.cuh"
#include "tma.cuh"

namespace wfe {
namespace {

// columns, level lanes, largest chunk, stages
struct PipeShape {
  int cx, kl, kch, nst;
};
constexpr PipeShape kPipeShapes[] = {{32, 16, 4, 2}, {16, 16, 4, 2}, {16, 16, 4, 3}};
constexpr int kNumPipeShapes = 3;
// a stage wait gives up after this much wall time (the loads take microseconds)
constexpr uint64_t kPipeWaitNs = 4000000000ull;

__host__ __device__ inline void pipe_box(int cx, int f, int nz, int* bx, int* by, int* bz) {
  *bx = (f == TC_U || f == TC_RTJX) ? cx + 4 : cx;
  *by = (f == TC_V || f == TC_RTJY) ? 2 : 1;
  *bz = f == TC_W ? nz + 1 : nz;
}

__host__ __device__ inline bool pipe_loaded(int f, bool moist, bool tpi, bool prof = false) {
  if (prof && pipe_prof_slot(f) >= 0) return false;
  if (f == TC_TPI) return tpi;
  if (f >= TC_QV) return moist;
  return true;
}

// Shared memory: 2 * NST mbarriers, NST stages of the loaded fields' boxes
// (each 128-byte aligned), then the row arrays A, B, C and D (D holds the
// solution w after the sweep; w at level 0 is written by the lane of level 0)
template <typename R>
struct PipeLayout {
  size_t field[TC_N];
  size_t stage0, stage_bytes, work, total;
  uint32_t tx_bytes;
  __host__ __device__ PipeLayout(int cx, int nz, int nst, bool moist, bool tpi, bool prof = false) {
    size_t o = 0;
    tx_bytes = 0;
    for (int f = 0; f < TC_N; ++f) {
      field[f] = 0;
      if (!pipe_loaded(f, moist, tpi, prof)) continue;
      int bx, by, bz;
      pipe_box(cx, f, nz, &bx, &by, &bz);
      const size_t b = (size_t)bx * by * bz * sizeof(R);
      field[f] = o;
      o += (b + 127) / 128 * 128;
      tx_bytes += (uint32_t)b;
    }
    stage_bytes = o;
    stage0 = 128;
    work = stage0 + (size_t)nst * stage_bytes;
    total = work + (size_t)4 * (nz + 1) * cx * sizeof(R);
  }
};

// The producer thread of a pipelined column CTA: for each of the CTA's tiles
// in order, wait until the consumers released the stage's previous tile,
// then stream the tile's boxes into the stage with bulk tensor loads (no
// multicast: the maps cover this GPU's own fields only).  Every wait is
// bounded; on a timeout it sets *err and stops issuing.
template <typename R, int CX, int NST, bool PROF = false>
__device__ __forceinline__ void pipe_produce(const PipeColParams<R>& p, const PipeLayout<R>& lay,
                                             unsigned char* smem_pipe, uint64_t* full, uint64_t* empty,
                                             int ntx, int ntiles) {
  const bool moist = p.a.p.moisture != 0;
  const bool has_tpi = p.has_tpi != 0;
  int n = 0, armed[NST];
  for (int s = 0; s < NST; ++s) armed[s] = -1;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++n) {
    const int s = n % NST, use = n / NST;
    // the consumers released this stage's previous tile
    if (use > 0 && !tma::mbar_wait_for(&empty[s], (use - 1) & 1, kPipeWaitNs)) {
      atomicExch(p.err, 1u);
      break;
    }
    tma::mbar_arrive_expect_tx(&full[s], lay.tx_bytes);
    armed[s] = use;
    unsigned char* stg = smem_pipe + lay.stage0 + (size_t)s * lay.stage_bytes;
    const int x = (t % ntx) * CX + kOX, y = t / ntx + kOY, z = kOZ;
    for (int f = 0; f < TC_N; ++f)
      if (pipe_loaded(f, moist, has_tpi, PROF))
        tma::load_3d(stg + lay.field[f], &p.map[f], x, y, z, &full[s]);
  }
  // loads this CTA armed must land before it exits (they have, unless the
  // consumers gave up early)
  for (int s = 0; s < NST; ++s)
    if (armed[s] >= 0) tma::mbar_wait_for(&full[s], armed[s] & 1, kPipeWaitNs);
}

template <typename R, int CX, int KL, int KCH, int NST, bool PROF>
__global__ void __launch_bounds__(CX * KL + 32, CX == 32 ? 1 : 2)
    k_acoustic_column_pipe(const __grid_constant__ PipeColParams<R> p) {
  extern __shared__ __align__(128) unsigned char smem_pipe[];
  constexpr int NC = CX * KL;  // consumer threads; the last warp produces
  // the consumers' named barrier counts whole warps, and the producer warp
  // holds no consumer
  static_assert(NC % 32 == 0, "consumer threads must fill whole warps");
  const AcouArgs<R>& a = p.a;
  const Layout& L = a.L;
  const int nz = L.nz;
  const bool moist = a.p.moisture != 0;
  const bool has_tpi = p.has_tpi != 0;
  const PipeLayout<R> lay(CX, nz, NST, moist, has_tpi, PROF);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_pipe);
  uint64_t* empty = full + NST;
  const int tid = threadIdx.x;
  const int ntx = (L.nx + CX - 1) / CX;
  const int ntiles = ntx * L.ny;
  if (tid == 0) {
    for (int s = 0; s < NST; ++s) {
      tma::mbar_init(&full[s], 1);
      tma::mbar_init(&empty[s], 1);
    }
    tma::fence_barrier_init();
  }
  __syncthreads();

  if (tid >= NC) {
    if (tid == NC) pipe_produce<R, CX, NST, PROF>(p, lay, smem_pipe, full, empty, ntx, ntiles);
    return;
  }

  // -------------------------------------------------------------- consumers
  const int tx = tid % CX, lane = tid / CX;
  const size_t n1 = (size_t)(nz + 1) * CX;
  R* sA = reinterpret_cast<R*>(smem_pipe + lay.work);
  R* sB = sA + n1;
  R* sC = sB + n1;
  R* sD = sC + n1;
  // (PROF) the coefficient fields' level values, once per CTA
  R* lvl_prof = sD + n1;
  if (PROF) {
    for (int q = tid; q < PF_N * (nz + 1); q += NC) lvl_prof[q] = p.prof[q];
    tma::named_sync(1, NC);
  }
  const R dtau = a.dtau;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const int pl = L.planei();
  const int ch = (nz + KL) / KL;
  const int klo = lane * ch;
  int n = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++n) {
    const int s = n % NST, use = n / NST;
    const bool ok = tma::mbar_wait_for(&full[s], use & 1, kPipeWaitNs);
    if (tma::named_or(1, NC, !ok)) {
      if (tid == 0) atomicExch(p.err, 1u);
      break;
    }
    const unsigned char* stg = smem_pipe + lay.stage0 + (size_t)s * lay.stage_bytes;
    auto fld = [&](int f) { return reinterpret_cast<const R*>(stg + lay.field[f]); };
    const R* sU = fld(TC_U);
    const R* sRX = fld(TC_RTJX);
    const R* sV = fld(TC_V);
    const R* sRY = fld(TC_RTJY);
    const R* sW = fld(TC_W);
    const R* sPI = fld(TC_PI);
    const R* sTH = fld(TC_TH);
    const R* sTW = fld(TC_TW);
    const R* sTTH = fld(TC_TTH);
    const R* sTPI = fld(TC_TPI);
    const R* sAW = fld(TC_AW);
    const R* sKT = fld(TC_KT3);
    const R* sTHBW = fld(TC_THBW);
    const R* sDTHB = fld(TC_DTHB);
    const R* sQV = fld(TC_QV);
    const R* sQC = fld(TC_QC);
    const R* sQR = fld(TC_QR);
    const R* sQVB = fld(TC_QVB);
#define UF(k, d) sU[(k) * (CX + 4) + tx + (d)]
#define RXF(k, d) (PROF ? lvl_prof[PF_RTJX * (nz + 1) + (k)] : sRX[(k) * (CX + 4) + tx + (d)])
#define VF(k, r) sV[((k) * 2 + (r)) * CX + tx]
#define RYF(k, r) (PROF ? lvl_prof[PF_RTJY * (nz + 1) + (k)] : sRY[((k) * 2 + (r)) * CX + tx])
#define CF(X, k) X[(k) * CX + tx]
#define PF(X, q, k) (PROF ? lvl_prof[(q) * (nz + 1) + (k)] : CF(X, k))
#define SQ(X, k) X[(size_t)(k) * CX + tx]
    const int i = (t % ntx) * CX + tx, j = t / ntx;
    const bool active = i < L.nx;
    const int c2d = L.at2i(active ? i : 0, j);
    const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
    const R invJ = (R)1 / J;
    const R mcx = mc * a.co.inv_dx, mcy = mc * a.co.inv_dy;
    const bool terrain = hxc != (R)0 || hyc != (R)0;
    R av[KCH + 2], sv[KCH + 2], P[KCH + 1], E[KCH + 1], th[KCH + 1], tt[KCH + 1], db[KCH + 1];
    if (active) {
      // phase 1 on levels klo-1 .. klo+ch
#pragma unroll
      for (int q = 0; q < KCH + 2; ++q) {
        const int k = klo - 1 + q;
        R avk = 0, svk = 0;
        if (q <= ch + 1 && k >= 1 && k < nz) {
          avk = PF(sAW, PF_AW, k);
          if (terrain) {
            R uw = (R)0.25 * (UF(k - 1, 0) + UF(k - 1, 1) + UF(k, 0) + UF(k, 1));
            R vw = (R)0.25 * (VF(k - 1, 0) + VF(k - 1, 1) + VF(k, 0) + VF(k, 1));
            svk = avk * (uw * hxc + vw * hyc) * a.co.fac_w[L.at1(k)];
          }
        }
        av[q] = avk;
        sv[q] = svk;
      }
      // phase 2 on levels klo-1 .. klo+ch-1
#pragma unroll
      for (int q = 0; q < KCH + 1; ++q) {
        const int k = klo - 1 + q;
        R pk = 0, ek = 0;
        if (q <= ch && k >= 0 && k < nz) {
          const int kk = L.at1(k);
          R Kt = PF(sKT, PF_KT3, k);
          R Dh = (RXF(k, 1) * UF(k, 1) - RXF(k, 0) * UF(k, 0)) * mcx +
                 (RYF(k, 1) * VF(k, 1) - RYF(k, 0) * VF(k, 0)) * mcy;
          R idz = a.co.inv_dzc[kk];
          R wk = CF(sW, k), wkp = CF(sW, k + 1);
          R tpi = has_tpi ? CF(sTPI, k) : (R)0;
          pk = CF(sPI, k) + dtau * tpi -
               dtau * Kt * (Dh - (sv[q + 1] - sv[q]) * idz + c2 * (av[q + 1] * wkp - av[q] * wk) * idz);
          ek = dtau * Kt * c1 * idz;
        }
        P[q] = pk;
        E[q] = ek;
      }
      // phase 3 on the inner levels of the chunk, and phase 5's inputs
#pragma unroll
      for (int q = 1; q < KCH + 1; ++q) {
        const int k = klo - 1 + q;
        if (q <= ch && k < nz) {
          th[q] = CF(sTH, k);
          tt[q] = CF(sTTH, k);
          db[q] = PF(sDTHB, PF_DTHB, k);
        }
        if (q <= ch && k >= 1 && k < nz) {
          const int kk = L.at1(k);
          const R iJdz = invJ * a.co.inv_dzw[kk];
          R thc = th[q], thm = CF(sTH, k - 1);
          R thbw = PF(sTHBW, PF_THBW, k);
          R thvw = thbw + (R)0.5 * (thm + thc);
          if (moist) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (CF(sQV, k - 1) + CF(sQV, k));
          R G = dtau * Phys<R>::cp * thvw * c1 * iJdz;
          R Em = E[q - 1], Ek = E[q];
          SQ(sA, k) = -G * Em * av[q - 1];
          SQ(sB, k) = (R)1 + G * av[q] * (Ek + Em);
          SQ(sC, k) = -G * Ek * av[q + 1];
          R buoy = Phys<R>::grav * (R)0.5 * (thm + thc) / thbw;
          if (moist) {
            R dqv = (R)0.5 * (CF(sQV, k - 1) + CF(sQV, k)) - (R)0.5 * (PF(sQVB, PF_QVB, k - 1) + PF(sQVB, PF_QVB, k));
            R qcr = (R)0.5 * (CF(sQC, k - 1) + CF(sQC, k)) + (R)0.5 * (CF(sQR, k - 1) + CF(sQR, k));
            buoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - qcr);
          }
          R RHS = CF(sW, k) + dtau * (buoy + CF(sTW, k)) -
                  dtau * Phys<R>::cp * thvw * c2 * (CF(sPI, k) - CF(sPI, k - 1)) * iJdz;
          SQ(sD, k) = RHS - G * (P[q] - P[q - 1]);
        }
      }
      if (lane == 0) {  // diagnostic surface w from the new u, v
        R us = (R)0.5 * (UF(0, 0) + UF(0, 1));
        R vs = (R)0.5 * (VF(0, 0) + VF(0, 1));
        SQ(sD, 0) = us * hxc + vs * hyc;
      }
    }
    tma::named_sync(1, NC);
    // every input of this tile is in registers or the row arrays: the
    // producer may refill the stage
    if (tid == 0) tma::mbar_arrive(&empty[s]);
    // phase 4: the Thomas sweep of the chunked kernel, one thread per column;
    // the solution overwrites D
    if (active && lane == 0) {
      R cprev = 0, dprev = 0;
      R Ak = SQ(sA, 1), Bk = SQ(sB, 1), Ck = SQ(sC, 1), Dk = SQ(sD, 1);
      for (int k = 1; k < nz; ++k) {
        R An = 0, Bn = 1, Cn = 0, Dn = 0;
        if (k + 1 < nz) {
          An = SQ(sA, k + 1);
          Bn = SQ(sB, k + 1);
          Cn = SQ(sC, k + 1);
          Dn = SQ(sD, k + 1);
        }
        R r, ck, dk;
        if (k == 1) {
          r = (R)1 / Bk;
          ck = Ck * r;
          dk = Dk * r;
        } else {
          r = (R)1 / (Bk - Ak * cprev);
          ck = Ck * r;
          dk = (Dk - Ak * dprev) * r;
        }
        SQ(sC, k) = ck;
        SQ(sD, k) = dk;
        cprev = ck;
        dprev = dk;
        Ak = An, Bk = Bn, Ck = Cn, Dk = Dn;
      }
      SQ(sD, nz) = 0;
      R wabove = 0;
      for (int k = nz - 1; k >= 1; --k) {
        R wk = SQ(sD, k) - SQ(sC, k) * wabove;
        SQ(sD, k) = wk;
        wabove = wk;
      }
    }
    tma::named_sync(1, NC);
    // phase 5 on the chunk's levels
    if (active) {
      const int c0 = L.ati(i, j, 0);
#pragma unroll
      for (int q = 1; q < KCH + 1; ++q) {
        const int k = klo - 1 + q;
        if (q > ch || k > nz) continue;
        const int c = c0 + k * pl;
        if (k < nz) {
          R wn = SQ(sD, k), wn1 = SQ(sD, k + 1);
          a.pi_next[c] = P[q] - E[q] * (av[q + 1] * wn1 - av[q] * wn);
          R wc = (R)0.5 * (wn + wn1);
          a.th_out[c] = th[q] + dtau * (tt[q] - wc * db[q]);
          a.w_out[c] = wn;
        } else {
          a.w_out[c] = 0;
        }
      }
    }
    // the next tile's rows overwrite the arrays phase 5 just read
    tma::named_sync(1, NC);
#undef UF
#undef RXF
#undef VF
#undef RYF
#undef CF
#undef PF
#undef SQ
  }
}

// The pipelined column with the parallel solve: the producer warp and the
// stage ring of k_acoustic_column_pipe, the phases and the solve of the
// parallel-solve column kernel (dyn_acou.cu: level lane p owns the levels
// p KCH .. p KCH + KCH - 1 in registers, identity rows pad the column,
// pcr_solve).  The consumers release a stage as soon as phases 1-3 have read
// it, so the next tile's boxes land while this tile is solved, and no lane
// waits for a serial sweep.  Every expression is the parallel-solve kernel's
// on the same values (from shared memory instead of global memory).
template <typename R, int CX, int KL, int KCH, int NST, bool PROF>
__global__ void __launch_bounds__(CX * KL + 32)
    k_acoustic_column_pipe_pcr(const __grid_constant__ PipeColParams<R> p) {
  extern __shared__ __align__(128) unsigned char smem_pipe[];
  constexpr int NC = CX * KL;  // consumer threads; the last warp produces
  // the consumers' named barrier counts whole warps, and the producer warp
  // holds no consumer
  static_assert(NC % 32 == 0, "consumer threads must fill whole warps");
  const AcouArgs<R>& a = p.a;
  const Layout& L = a.L;
  const int nz = L.nz;
  const bool moist = a.p.moisture != 0;
  const bool has_tpi = p.has_tpi != 0;
  const PipeLayout<R> lay(CX, nz, NST, moist, has_tpi, PROF);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_pipe);
  uint64_t* empty = full + NST;
  const int tid = threadIdx.x;
  const int ntx = (L.nx + CX - 1) / CX;
  const int ntiles = ntx * L.ny;
  if (tid == 0) {
    for (int s = 0; s < NST; ++s) {
      tma::mbar_init(&full[s], 1);
      tma::mbar_init(&empty[s], 1);
    }
    tma::fence_barrier_init();
  }
  __syncthreads();
  if (tid >= NC) {
    if (tid == NC) pipe_produce<R, CX, NST, PROF>(p, lay, smem_pipe, full, empty, ntx, ntiles);
    return;
  }

  // -------------------------------------------------------------- consumers
  const int tx = tid % CX, lane = tid / CX;
  R* work = reinterpret_cast<R*>(smem_pipe + lay.work);
  // the per-level tables every tile reads, once per CTA: 1/dzc, 1/dzw and the
  // terrain factor of the w levels, at level k, and (PROF) the coefficient
  // fields' level values
  R* lvl_idzc = work + kPcrWork * NC;
  R* lvl_idzw = lvl_idzc + (nz + 1);
  R* lvl_facw = lvl_idzw + (nz + 1);
  R* lvl_prof = lvl_facw + (nz + 1);
  for (int k = tid; k <= nz; k += NC) {
    lvl_idzc[k] = a.co.inv_dzc[L.at1(k)];
    lvl_idzw[k] = a.co.inv_dzw[L.at1(k)];
    lvl_facw[k] = a.co.fac_w[L.at1(k)];
  }
  if (PROF)
    for (int q = tid; q < PF_N * (nz + 1); q += NC) lvl_prof[q] = p.prof[q];
  const R dtau = a.dtau;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const int pl = L.planei();
  const int klo = lane * KCH;
  auto csync = [] { tma::named_sync(1, NC); };
  csync();
  int n = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++n) {
    const int s = n % NST, use = n / NST;
    // the column's metric, loaded while the tile's boxes may still be landing
    const int i = (t % ntx) * CX + tx, j = t / ntx;
    const bool active = i < L.nx;
    const int c2d = L.at2i(active ? i : 0, j);
    const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
    const bool ok = tma::mbar_wait_for(&full[s], use & 1, kPipeWaitNs);
    if (tma::named_or(1, NC, !ok)) {
      if (tid == 0) atomicExch(p.err, 1u);
      break;
    }
    const unsigned char* stg = smem_pipe + lay.stage0 + (size_t)s * lay.stage_bytes;
    auto fld = [&](int f) { return reinterpret_cast<const R*>(stg + lay.field[f]); };
    const R* sU = fld(TC_U);
    const R* sRX = fld(TC_RTJX);
    const R* sV = fld(TC_V);
    const R* sRY = fld(TC_RTJY);
    const R* sW = fld(TC_W);
    const R* sPI = fld(TC_PI);
    const R* sTH = fld(TC_TH);
    const R* sTW = fld(TC_TW);
    const R* sTTH = fld(TC_TTH);
    const R* sTPI = fld(TC_TPI);
    const R* sAW = fld(TC_AW);
    const R* sKT = fld(TC_KT3);
    const R* sTHBW = fld(TC_THBW);
    const R* sDTHB = fld(TC_DTHB);
    const R* sQV = fld(TC_QV);
    const R* sQC = fld(TC_QC);
    const R* sQR = fld(TC_QR);
    const R* sQVB = fld(TC_QVB);
#define UF(k, d) sU[(k) * (CX + 4) + tx + (d)]
#define RXF(k, d) (PROF ? lvl_prof[PF_RTJX * (nz + 1) + (k)] : sRX[(k) * (CX + 4) + tx + (d)])
#define VF(k, r) sV[((k) * 2 + (r)) * CX + tx]
#define RYF(k, r) (PROF ? lvl_prof[PF_RTJY * (nz + 1) + (k)] : sRY[((k) * 2 + (r)) * CX + tx])
#define CF(X, k) X[(k) * CX + tx]
#define PF(X, q, k) (PROF ? lvl_prof[(q) * (nz + 1) + (k)] : CF(X, k))
    const R invJ = (R)1 / J;
    const R mcx = mc * a.co.inv_dx, mcy = mc * a.co.inv_dy;
    const bool terrain = hxc != (R)0 || hyc != (R)0;
    R av[KCH + 2], sv[KCH + 2], P[KCH + 1], E[KCH + 1], th[KCH + 1], tt[KCH + 1], db[KCH + 1];
    R Ar[KCH + 1], Br[KCH + 1], Cr[KCH + 1], Dr[KCH + 1];
    R wsurf = 0;
#pragma unroll
    for (int q = 0; q < KCH + 1; ++q) Ar[q] = 0, Br[q] = 1, Cr[q] = 0, Dr[q] = 0;
    if (active) {
      // phase 1 on levels klo-1 .. klo+KCH
#pragma unroll
      for (int q = 0; q < KCH + 2; ++q) {
        const int k = klo - 1 + q;
        R avk = 0, svk = 0;
        if (k >= 1 && k < nz) {
          avk = PF(sAW, PF_AW, k);
          if (terrain) {
            R uw = (R)0.25 * (UF(k - 1, 0) + UF(k - 1, 1) + UF(k, 0) + UF(k, 1));
            R vw = (R)0.25 * (VF(k - 1, 0) + VF(k - 1, 1) + VF(k, 0) + VF(k, 1));
            svk = avk * (uw * hxc + vw * hyc) * lvl_facw[k];
          }
        }
        av[q] = avk;
        sv[q] = svk;
      }
      // phase 2 on levels klo-1 .. klo+KCH-1
#pragma unroll
      for (int q = 0; q < KCH + 1; ++q) {
        const int k = klo - 1 + q;
        R pk = 0, ek = 0;
        if (k >= 0 && k < nz) {
          R Kt = PF(sKT, PF_KT3, k);
          R Dh = (RXF(k, 1) * UF(k, 1) - RXF(k, 0) * UF(k, 0)) * mcx +
                 (RYF(k, 1) * VF(k, 1) - RYF(k, 0) * VF(k, 0)) * mcy;
          R idz = lvl_idzc[k];
          R wk = CF(sW, k), wkp = CF(sW, k + 1);
          R tpi = has_tpi ? CF(sTPI, k) : (R)0;
          pk = CF(sPI, k) + dtau * tpi -
               dtau * Kt * (Dh - (sv[q + 1] - sv[q]) * idz + c2 * (av[q + 1] * wkp - av[q] * wk) * idz);
          ek = dtau * Kt * c1 * idz;
        }
        P[q] = pk;
        E[q] = ek;
      }
      // phase 3: rows of the inner levels, and phase 5's inputs
#pragma unroll
      for (int q = 1; q < KCH + 1; ++q) {
        const int k = klo - 1 + q;
        th[q] = tt[q] = db[q] = 0;
        if (k < nz) {
          th[q] = CF(sTH, k);
          tt[q] = CF(sTTH, k);
          db[q] = PF(sDTHB, PF_DTHB, k);
        }
        if (k >= 1 && k < nz) {
          const R iJdz = invJ * lvl_idzw[k];
          R thc = th[q], thm = CF(sTH, k - 1);
          R thbw = PF(sTHBW, PF_THBW, k);
          R thvw = thbw + (R)0.5 * (thm + thc);
          if (moist) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (CF(sQV, k - 1) + CF(sQV, k));
          R G = dtau * Phys<R>::cp * thvw * c1 * iJdz;
          R Em = E[q - 1], Ek = E[q];
          Ar[q] = -G * Em * av[q - 1];
          Br[q] = (R)1 + G * av[q] * (Ek + Em);
          Cr[q] = -G * Ek * av[q + 1];
          R buoy = Phys<R>::grav * (R)0.5 * (thm + thc) / thbw;
          if (moist) {
            R dqv = (R)0.5 * (CF(sQV, k - 1) + CF(sQV, k)) - (R)0.5 * (PF(sQVB, PF_QVB, k - 1) + PF(sQVB, PF_QVB, k));
            R qcr = (R)0.5 * (CF(sQC, k - 1) + CF(sQC, k)) + (R)0.5 * (CF(sQR, k - 1) + CF(sQR, k));
            buoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - qcr);
          }
          R RHS = CF(sW, k) + dtau * (buoy + CF(sTW, k)) -
                  dtau * Phys<R>::cp * thvw * c2 * (CF(sPI, k) - CF(sPI, k - 1)) * iJdz;
          Dr[q] = RHS - G * (P[q] - P[q - 1]);
        }
      }
      if (lane == 0) {  // diagnostic surface w from the new u, v
        R us = (R)0.5 * (UF(0, 0) + UF(0, 1));
        R vs = (R)0.5 * (VF(0, 0) + VF(0, 1));
        wsurf = us * hxc + vs * hyc;
      }
    }
#undef UF
#undef RXF
#undef VF
#undef RYF
#undef CF
#undef PF
    // every input of this tile is in registers: the producer may refill the
    // stage (the barrier also ends the previous tile's use of the work area)
    csync();
    if (tid == 0) tma::mbar_arrive(&empty[s]);
    PcrLane<R, KCH> sol;
    pcr_solve<R, CX, KL, KCH>(Ar, Br, Cr, Dr, work, tx, lane, csync, sol);
    // phase 5: pi', theta', w of the lane's levels
    if (active) {
      const int c0 = L.ati(i, j, 0);
      R wl[KCH + 2];  // w at the lane's levels and the level above them
#pragma unroll
      for (int q = 1; q < KCH; ++q) wl[q] = sol.Gx[q] + sol.Ax[q] * sol.yprev + sol.Bx[q] * sol.y;
      wl[KCH] = sol.y;
      wl[KCH + 1] = sol.gn + sol.an * sol.y + sol.bn * sol.ynext;
      if (lane == 0) wl[1] = wsurf;  // level 0: the diagnostic surface w
#pragma unroll
      for (int q = 1; q < KCH + 1; ++q) {
        const int k = klo - 1 + q;
        if (k > nz) continue;
        const int c = c0 + k * pl;
        if (k == nz) {
          a.w_out[c] = 0;
          continue;
        }
        const R wn = wl[q], wn1 = k + 1 >= nz ? (R)0 : wl[q + 1];
        a.pi_next[c] = P[q] - E[q] * (av[q + 1] * wn1 - av[q] * wn);
        R wc = (R)0.5 * (wn + wn1);
        a.th_out[c] = th[q] + dtau * (tt[q] - wc * db[q]);
        a.w_out[c] = wn;
      }
    }
  }
}

// columns, level lanes, levels per lane, stages (14 lanes of 3 levels hold
// the 41 rows of a 40-level column with one identity row instead of seven)
constexpr PipeShape kPipePcrShapes[] = {{16, 16, 3, 2}, {8, 16, 3, 2}, {8, 16, 3, 3}, {16, 14, 3, 2}};
constexpr int kNumPipePcrShapes = 4;

template <typename R, int F, bool PROF>
struct PipePcrKernel {
  static constexpr PipeShape S = kPipePcrShapes[F];
  static constexpr auto fn = k_acoustic_column_pipe_pcr<R, S.cx, S.kl, S.kch, S.nst, PROF>;
};

template <typename R, bool PROF>
const void* pipe_pcr_fn(int f) {
  switch (f) {
    case 0: return reinterpret_cast<const void*>(PipePcrKernel<R, 0, PROF>::fn);
    case 1: return reinterpret_cast<const void*>(PipePcrKernel<R, 1, PROF>::fn);
    case 2: return reinterpret_cast<const void*>(PipePcrKernel<R, 2, PROF>::fn);
    default: return reinterpret_cast<const void*>(PipePcrKernel<R, 3, PROF>::fn);
  }
}

template <typename R>
const void* pipe_pcr_fn(int f, bool prof) {
  return prof ? pipe_pcr_fn<R, true>(f) : pipe_pcr_fn<R, false>(f);
}

template <typename R, bool PROF>
void launch_pipe_pcr(int f, int grid, int threads, size_t sm, cudaStream_t st, const PipeColParams<R>& p) {
  switch (f) {
    case 0: PipePcrKernel<R, 0, PROF>::fn<<<grid, threads, sm, st>>>(p); break;
    case 1: PipePcrKernel<R, 1, PROF>::fn<<<grid, threads, sm, st>>>(p); break;
    case 2: PipePcrKernel<R, 2, PROF>::fn<<<grid, threads, sm, st>>>(p); break;
    default: PipePcrKernel<R, 3, PROF>::fn<<<grid, threads, sm, st>>>(p); break;
  }
}

template <typename R, int F, bool PROF>
struct PipeKernel {
  static constexpr PipeShape S = kPipeShapes[F];
  static constexpr auto fn = k_acoustic_column_pipe<R, S.cx, S.kl, S.kch, S.nst, PROF>;
};

template <typename R, bool PROF>
const void* pipe_fn(int f) {
  switch (f) {
    case 0: return reinterpret_cast<const void*>(PipeKernel<R, 0, PROF>::fn);
    case 1: return reinterpret_cast<const void*>(PipeKernel<R, 1, PROF>::fn);
    default: return reinterpret_cast<const void*>(PipeKernel<R, 2, PROF>::fn);
  }
}

template <typename R>
const void* pipe_fn(int f, bool prof) {
  return prof ? pipe_fn<R, true>(f) : pipe_fn<R, false>(f);
}

template <typename R, bool PROF>
void launch_pipe(int f, int grid, int threads, size_t sm, cudaStream_t st, const PipeColParams<R>& p) {
  switch (f) {
    case 0: PipeKernel<R, 0, PROF>::fn<<<grid, threads, sm, st>>>(p); break;
    case 1: PipeKernel<R, 1, PROF>::fn<<<grid, threads, sm, st>>>(p); break;
    default: PipeKernel<R, 2, PROF>::fn<<<grid, threads, sm, st>>>(p); break;
  }
}

// resident CTAs of kernel fn (threads per CTA, `smem` bytes) on the whole
// device: the persistent grid (cached)
int pipe_grid_limit(const void* fn, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<std::pair<int, const void*>, size_t>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(std::make_pair(dev, fn), smem);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int sms = 0, occ = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem) != cudaSuccess) return 0;
  return cache[key] = sms * occ;
}

}  // namespace

int acoustic_pipe_shapes() { return kNumPipeShapes; }

void acoustic_pipe_box(int shape, int f, int nz, int* bx, int* by, int* bz) {
  pipe_box(kPipeShapes[shape].cx, f, nz, bx, by, bz);
}

template <typename R>
size_t acoustic_pipe_smem(int shape, int nz, bool moist, bool tpi, bool prof) {
  if (shape < 0 || shape >= kNumPipeShapes) return 0;
  const PipeShape& S = kPipeShapes[shape];
  if (nz + 1 > S.kl * S.kch || nz + 1 > 256) return 0;  // chunks; a box extent is <= 256
  const size_t t = PipeLayout<R>(S.cx, nz, S.nst, moist, tpi, prof).total +
                   (prof ? (size_t)PF_N * (nz + 1) * sizeof(R) : 0);
  return t <= 227 * 1024 ? t : 0;
}

template <typename R>
size_t acoustic_pipe_pcr_smem(int shape, int nz, bool moist, bool tpi, bool prof) {
  if (shape < 0 || shape >= kNumPipePcrShapes) return 0;
  const PipeShape& S = kPipePcrShapes[shape];
  if (nz + 1 > S.kl * S.kch || nz + 1 > 256) return 0;  // rows; a box extent is <= 256
  const size_t tables = (size_t)(3 + (prof ? PF_N : 0)) * (nz + 1);
  const size_t t = PipeLayout<R>(S.cx, nz, S.nst, moist, tpi, prof).work +
                   ((size_t)kPcrWork * S.kl * S.cx + tables) * sizeof(R);
  return t <= 227 * 1024 ? t : 0;
}

template <typename R>
int prepare_acoustic_pipe(int nz) {
  bool any = false;
  // kinds: the Thomas pipeline and the parallel-solve pipeline, each with
  // boxes for every field (prof 0) and with the level tables (prof 1)
  for (int pcr = 0; pcr < 2; ++pcr)
    for (int prof = 0; prof < 2; ++prof)
      for (int f = 0; f < (pcr ? kNumPipePcrShapes : kNumPipeShapes); ++f) {
        size_t sm = 0;
        for (int moist = 0; moist < 2; ++moist)
          for (int tpi = 0; tpi < 2; ++tpi) {
            const size_t t = pcr ? acoustic_pipe_pcr_smem<R>(f, nz, moist != 0, tpi != 0, prof != 0)
                                 : acoustic_pipe_smem<R>(f, nz, moist != 0, tpi != 0, prof != 0);
            if (t > sm) sm = t;
          }
        if (!sm) continue;
        if (raise_smem_limit(pcr ? pipe_pcr_fn<R>(f, prof != 0) : pipe_fn<R>(f, prof != 0), sm) != cudaSuccess)
          return 1;
        any = true;
      }
  return any ? 0 : 2;
}

int acoustic_pipe_pcr_shapes() { return kNumPipePcrShapes; }

void acoustic_pipe_pcr_box(int shape, int f, int nz, int* bx, int* by, int* bz) {
  pipe_box(kPipePcrShapes[shape].cx, f, nz, bx, by, bz);
}

template <typename R>
int launch_acoustic_column_pipe_pcr(const PipeColParams<R>& p, int f, cudaStream_t st) {
  const bool prof = p.prof != nullptr;
  const size_t sm = acoustic_pipe_pcr_smem<R>(f, p.a.L.nz, p.a.p.moisture != 0, p.has_tpi != 0, prof);
  if (!sm) return 2;
  const PipeShape& S = kPipePcrShapes[f];
  const int ntiles = (p.a.L.nx + S.cx - 1) / S.cx * p.a.L.ny;
  const int threads = S.cx * S.kl + 32;
  const int lim = pipe_grid_limit(pipe_pcr_fn<R>(f, prof), threads, sm);
  if (lim <= 0) return 2;
  const int grid = ntiles < lim ? ntiles : lim;
  if (prof) launch_pipe_pcr<R, true>(f, grid, threads, sm, st, p);
  else launch_pipe_pcr<R, false>(f, grid, threads, sm, st, p);
  return 0;
}

template <typename R>
int launch_acoustic_column_pipe(const PipeColParams<R>& p, int f, cudaStream_t st) {
  const bool prof = p.prof != nullptr;
  const size_t sm = acoustic_pipe_smem<R>(f, p.a.L.nz, p.a.p.moisture != 0, p.has_tpi != 0, prof);
  if (!sm) return 2;
  const PipeShape& S = kPipeShapes[f];
  const int ntiles = (p.a.L.nx + S.cx - 1) / S.cx * p.a.L.ny;
  const int threads = S.cx * S.kl + 32;
  const int lim = pipe_grid_limit(pipe_fn<R>(f, prof), threads, sm);
  if (lim <= 0) return 2;
  const int grid = ntiles < lim ? ntiles : lim;
  if (prof) launch_pipe<R, true>(f, grid, threads, sm, st, p);
  else launch_pipe<R, false>(f, grid, threads, sm, st, p);
  return 0;
}

#define WFE_INST(R)                                                              \
  template size_t acoustic_pipe_smem<R>(int, int, bool, bool, bool);             \
  template size_t acoustic_pipe_pcr_smem<R>(int, int, bool, bool, bool);         \
  template int prepare_acoustic_pipe<R>(int);                                    \
  template int launch_acoustic_column_pipe<R>(const PipeColParams<R>&, int, cudaStream_t); \
  template int launch_acoustic_column_pipe_pcr<R>(const PipeColParams<R>&, int, cudaStream_t);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
