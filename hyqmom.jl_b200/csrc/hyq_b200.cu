// libhyqmom_b200.so: kernels and C-ABI of the HyQMOM explicit step on B200.
//
// One step = thirteen launches on the context stream, captured once in a CUDA
// graph and replayed:
//   phase A      five per-cell kernels (k_phase_A.cu): closure +
//                realizability, x, y and z flux-Jacobian eigenvalues with
//                their corrections, closure of the realized moments with
//                fluxes and the 1-D closure speeds; writes Fx, Fy, Fz, the
//                realized state and 6 speeds, and a NaN-propagating
//                per-block max |speed| (src/simulation_runner.jl:352-383)
//   k_cfl        one block: global max -> dt, t += dt, nn += 1 on the device
//                (src/simulation_runner.jl:402-433, 496)
//   k_hll        per cell, all 35 moments: x, y, z HLL updates with pas_HLL's copy
//                boundary handling, combined as Mx + My + Mz - 2M
//                (src/numerics/apply_flux_update_3d.jl:30-213,
//                 src/numerics/pas_HLL.jl:238-298, flux_HLL.jl:318-330,
//                 src/simulation_runner.jl:498-520)
//   phase EF     per-cell kernels (k_phase_EF.cu): realizability pass, with
//                the eigen corrections of listed cells in their own pass,
//                and BGK collision (src/simulation_runner.jl:526-557)
// The loop predicate `t < tmax && nn < nnmax` is evaluated on the device, so
// any number of steps can be queued without a host round trip.
//
// State: moment-major SoA, M[c + N*n], c = i + Nx*(j + Ny*k) (Julia order).
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>
#include <algorithm>
#include "hyq_cell.cuh"
#include "hyq_step.cuh"
#include "../../include/hyqmom.h"

using namespace hyq;
using namespace hyqk;

namespace {

__device__ __forceinline__ void cfl_body(const double* __restrict__ blockmax, const StepConst& sc, DevClock* clk) {
  const bool active = (clk->t < sc.tmax) && (clk->nn < sc.nnmax);
  __syncthreads();
  if (!active) {
    if (threadIdx.x == 0) clk->active = 0;
    return;
  }
  double v = 0.0;
  for (int b = threadIdx.x; b < sc.nblocksA; b += 1024) v = nanmax(v, blockmax[b]);
  const double vmax = block_nanmax<1024>(v);
  if (threadIdx.x == 0) {
    // A non-finite wave speed: the reference's eigvals would throw here
    // (src/numerics/eigenvalues6z_hyperbolic_3D.jl:108); the step still runs
    // with the NaN dt exactly as the Julia arithmetic would, and the status
    // word records the step at which it happened.
    if (!(vmax == vmax) || isinf(vmax)) { if (clk->status == 0) clk->status = (int)(clk->nn + 1); }
    double dt = jmin(sc.CFL * jmin(jmin(sc.dx, sc.dy), sc.dz) / vmax, jmin(sc.dtmax, sc.Kn));
    dt = jmin(dt, sc.tmax - clk->t);
    clk->vmax = vmax;
    clk->dt = dt;
    clk->t = clk->t + dt;
    clk->nn = clk->nn + 1;
    clk->active = 1;
  }
}
__global__ void __launch_bounds__(1024) k_cfl(const double* __restrict__ blockmax, const StepConst sc, DevClock* clk) {
  cfl_body(blockmax, sc, clk);
}
// fused batch: one block per member
__global__ void __launch_bounds__(1024) k_cfl_b(const Batch bt) {
  const Dom& d = bt.dom[blockIdx.x];
  const StepConst sc = d.sc;
  cfl_body(d.buf[DB_BMAX], sc, d.clk);
}

// The CFL reduction split for a domain decomposed over ranks: the local
// NaN-propagating max |speed| goes to xchg = {max over non-NaN, NaN flag},
// which the caller reduces with MAX over the ranks in place; k_cfl_global then
// takes dt from the global value exactly as k_cfl does from its own.
__global__ void __launch_bounds__(1024) k_vmax_local(const double* __restrict__ blockmax, const StepConst sc, const DevClock* clk,
                                                     double* xchg) {
  const bool active = (clk->t < sc.tmax) && (clk->nn < sc.nnmax);
  double v = 0.0;
  if (active)
    for (int b = threadIdx.x; b < sc.nblocksA; b += 1024) v = nanmax(v, blockmax[b]);
  const double vmax = block_nanmax<1024>(v);
  if (threadIdx.x == 0) {
    const bool nan = !(vmax == vmax);
    xchg[0] = nan ? 0.0 : vmax;
    xchg[1] = nan ? 1.0 : 0.0;
  }
}
__global__ void k_cfl_global(const double* xchg, const StepConst sc, DevClock* clk) {
  const bool active = (clk->t < sc.tmax) && (clk->nn < sc.nnmax);
  if (!active) { clk->active = 0; return; }
  const double vmax = xchg[1] > 0.0 ? __longlong_as_double(0x7ff8000000000000LL) : xchg[0];
  if (!(vmax == vmax) || isinf(vmax)) { if (clk->status == 0) clk->status = (int)(clk->nn + 1); }
  double dt = jmin(sc.CFL * jmin(jmin(sc.dx, sc.dy), sc.dz) / vmax, jmin(sc.dtmax, sc.Kn));
  dt = jmin(dt, sc.tmax - clk->t);
  clk->vmax = vmax;
  clk->dt = dt;
  clk->t = clk->t + dt;
  clk->nn = clk->nn + 1;
  clk->active = 1;
}

// pas_HLL along one line of Np cells (stride `st`, line start `base`) for the
// cell at position i of the line.  Its update reads the clamped cell ip and
// its two neighbours only (cells L = ip-1, C = ip, R = ip+1); everything
// that does not depend on the moment -- the HLL speeds of the two faces,
// whether W* is formed, and which of L, C, R the boundary rules substitute
// -- is resolved once per cell.
struct HllFace {
  double l1, l2;
  double rinv;              // 1 / (l1 - l2), for div_by
  bool w;                   // W* formed (|l1 - l2| > 1e-10)
  bool zero;                // face 0: zero speeds in the dissipation term
};
struct HllLine {
  long long base;           // offset of cell L
  int st;
  bool two;                 // Np == 2: pas_HLL returns [M2, M2]
  bool sh0;                 // ip == 1: face ip-1 uses W*[1] and F[1] (cell C)
  bool sh1;                 // ip + 1 == Np - 1: face ip uses F[Np-2] (cell C)
  double r;                 // dt / ds
  HllFace f0, f1;           // faces ip-1 and ip
};

__device__ __forceinline__ HllFace hll_face(const double* __restrict__ vmin, const double* __restrict__ vmax, long long base, int st, int j) {
  HllFace f;
  const int jj = j < 1 ? 1 : j;  // face 0 uses W*[1] with zero speeds
  const double a = vmin[base + st * jj], b = vmin[base + st * (jj + 1)];
  const double c = vmax[base + st * jj], d = vmax[base + st * (jj + 1)];
  f.l1 = jmin(a, b);
  f.l2 = jmax(c, d);
  f.w = fabs(f.l1 - f.l2) > 1e-10;
  f.rinv = 1.0 / (f.l1 - f.l2);
  f.zero = (j == 0);
  return f;
}

__device__ __forceinline__ HllLine hll_setup(const double* __restrict__ vmin, const double* __restrict__ vmax, long long base, int st,
                                             int Np, int i, double r) {
  HllLine L;
  L.st = st; L.r = r;
  L.two = (Np == 2);
  if (L.two) { L.base = base; L.sh0 = L.sh1 = false; return L; }
  const int ip = i < 1 ? 1 : (i > Np - 2 ? Np - 2 : i);
  L.base = base + (long long)st * (ip - 1);
  L.sh0 = (ip == 1);
  L.sh1 = (ip + 1 > Np - 2);
  L.f0 = hll_face(vmin, vmax, base, st, ip - 1);
  L.f1 = hll_face(vmin, vmax, base, st, ip);
  return L;
}

// flux_HLL at one face for one moment from the W* pair (mj, mj1, fj, fj1),
// the boundary-modified fluxes (Fa, Fb) and the face's cells (Ma_, Mb)
__device__ __forceinline__ double hll_flux(const HllFace& f, double mj, double mj1, double fj, double fj1, double Fa, double Fb, double Ma_,
                                           double Mb) {
  double ws = 0.0;
  if (f.w) {
    // the two divisions by l1 - l2 of the reference, through the face's
    // reciprocal (div_by returns the IEEE quotient bit for bit)
    const double d = f.l1 - f.l2;
    ws = div_by(f.l1 * mj - f.l2 * mj1, d, f.rinv) - div_by(fj - fj1, d, f.rinv);
  }
  // |lleft|, |lright| of the face (zero at face 0)
  const double al = f.zero ? 0.0 : fabs(f.l1), ar = f.zero ? 0.0 : fabs(f.l2);
  return 0.5 * (Fa + Fb) - 0.5 * (al * (ws - Ma_) - ar * (ws - Mb));
}

// The x, y or z update of one moment of the cell (pas_HLL for that line);
// M, F already offset to the moment.
// Mp, Fp: the moment and flux at cell L of the line (or at the line start
// when Np == 2), neighbours mst and fst apart (global memory or shared tiles).
__device__ __forceinline__ double hll_update_at(const double* Mp, const double* Fp, long long mst, long long fst, const HllLine& L) {
  if (L.two) return Mp[mst];
  const double mL = Mp[0], mC = Mp[mst], mR = Mp[2 * mst];
  const double fL = Fp[0], fC = Fp[fst], fR = Fp[2 * fst];
  const double f1 = hll_flux(L.f1, mC, mR, fC, fR, fC, L.sh1 ? fC : fR, mC, mR);
  const double f0 = L.sh0 ? hll_flux(L.f0, mC, mR, fC, fR, fC, fC, mL, mC) : hll_flux(L.f0, mL, mC, fL, fC, fL, fC, mL, mC);
  return mC - L.r * (f1 - f0);
}
__device__ __forceinline__ double hll_update(const double* __restrict__ M, const double* __restrict__ F, const HllLine& L) {
  return hll_update_at(M + L.base, F + L.base, L.st, L.st, L);
}

// One thread per cell and moment group: the face speeds of the x, y and z
// lines are resolved once, then the group's moments are updated in turn
// (coalesced along x).  GROUPS blocks cover the same BS cells, one group of
// moments each (consecutive blocks, so that they share the speed reads in
// L2); each moment's arithmetic is the same in every launch shape.
#ifndef HQ_MINB_HLL
#define HQ_MINB_HLL 4
#endif
template <int BS, int GROUPS>
__device__ __forceinline__ void hll_body(const double* __restrict__ M, const double* __restrict__ Fx, const double* __restrict__ Fy,
                                         const double* __restrict__ Fz, const double* __restrict__ vp, double* __restrict__ Mout,
                                         const StepConst& sc, const DevClock* clk, int bid) {
  if (!clk->active) return;
  const long long N = sc.N;
  const int grp = GROUPS == 1 ? 0 : bid % GROUPS;
  const long long c = (long long)(GROUPS == 1 ? bid : bid / GROUPS) * BS + threadIdx.x;
  if (c >= N) return;
  const double dt = clk->dt;
  const int Nx = sc.Nx, Ny = sc.Ny, Nz = sc.Nz;
  const int i = int(c % Nx);
  const int j = int((c / Nx) % Ny);
  const int k = int(c / ((long long)Nx * Ny));
  if (GROUPS == 1) {
    // all 35 moments: the three lines resolved together, one moment at a time
    const HllLine X = hll_setup(vp, vp + N, c - i, 1, Nx, i, dt / sc.dx);
    const HllLine Y = hll_setup(vp + 2 * N, vp + 3 * N, c - (long long)j * Nx, Nx, Ny, j, dt / sc.dy);
    HllLine Z;
    if (Nz > 1) Z = hll_setup(vp + 4 * N, vp + 5 * N, c - (long long)k * Nx * Ny, Nx * Ny, Nz, k, dt / sc.dz);
#pragma unroll 1
    for (int n = 0; n < 35; ++n) {
      const long long mo = N * n;
      const double* Mn = M + mo;
      const double mx = hll_update(Mn, Fx + mo, X);
      const double my = hll_update(Mn, Fy + mo, Y);
      const double mz = (Nz == 1) ? Mn[c] : hll_update(Mn, Fz + mo, Z);
      Mout[c + mo] = mx + my + mz - 2.0 * Mn[c];
    }
    return;
  }
  // a group of K moments: one line at a time over the group (fewer live
  // registers), the sums formed in the same order, ((mx + my) + mz) - 2 M
  constexpr int K = (35 + GROUPS - 1) / GROUPS;
  const int n0 = (35 * grp) / GROUPS, n1 = (35 * (grp + 1)) / GROUPS;
  double acc[K];
  {
    const HllLine X = hll_setup(vp, vp + N, c - i, 1, Nx, i, dt / sc.dx);
#pragma unroll
    for (int q = 0; q < K; ++q)
      if (n0 + q < n1) acc[q] = hll_update(M + N * (n0 + q), Fx + N * (n0 + q), X);
  }
  {
    const HllLine Y = hll_setup(vp + 2 * N, vp + 3 * N, c - (long long)j * Nx, Nx, Ny, j, dt / sc.dy);
#pragma unroll
    for (int q = 0; q < K; ++q)
      if (n0 + q < n1) acc[q] = acc[q] + hll_update(M + N * (n0 + q), Fy + N * (n0 + q), Y);
  }
  HllLine Z;
  if (Nz > 1) Z = hll_setup(vp + 4 * N, vp + 5 * N, c - (long long)k * Nx * Ny, Nx * Ny, Nz, k, dt / sc.dz);
#pragma unroll
  for (int q = 0; q < K; ++q)
    if (n0 + q < n1) {
      const long long mo = N * (n0 + q);
      const double* Mn = M + mo;
      const double mz = (Nz == 1) ? Mn[c] : hll_update(Mn, Fz + mo, Z);
      Mout[c + mo] = acc[q] + mz - 2.0 * Mn[c];
    }
}
template <int BS, int GROUPS, int MINB = HQ_MINB_HLL * 256 / BS>
__global__ void __launch_bounds__(BS, MINB) k_hll(const double* __restrict__ M, const double* __restrict__ Fx,
                                                                    const double* __restrict__ Fy, const double* __restrict__ Fz,
                                                                    const double* __restrict__ vp, double* __restrict__ Mout,
                                                                    const StepConst sc, const DevClock* clk) {
  hll_body<BS, GROUPS>(M, Fx, Fy, Fz, vp, Mout, sc, clk, blockIdx.x);
}
template <int BS, int GROUPS, int MINB = HQ_MINB_HLL * 256 / BS>
__global__ void __launch_bounds__(BS, MINB) k_hll_b(const Batch bt) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  hll_body<BS, GROUPS>(d.buf[DB_M], d.buf[DB_FX], d.buf[DB_FY], d.buf[DB_FZ], d.buf[DB_VP], d.buf[DB_MTMP], sc, d.clk,
                       blockIdx.x - __ldg(bt.blk0 + m));
}
// The HLL sweep on 32 x TY cell tiles of one layer, one group of five
// moments per block: the group's M (with two cells of halo along x and y),
// Fx and Fy tiles are staged in shared memory once, then one line of faces
// at a time reads its three cells from there (z from global memory), the
// sums formed in the same order as the per-cell kernels, ((mx + my) + mz) -
// 2 M, from the same values.
constexpr int HT_X = 32, HT_K = 5, HT_G = 7;
template <int TY>
__device__ __forceinline__ void hll_tile_body(const double* __restrict__ M, const double* __restrict__ Fx, const double* __restrict__ Fy,
                                              const double* __restrict__ Fz, const double* __restrict__ vp, double* __restrict__ Mout,
                                              const StepConst& sc, const DevClock* clk, int bid) {
  constexpr int MX = HT_X + 4, MY = TY + 4, SZM = MY * MX, SZX = TY * MX, SZY = MY * HT_X, BS = HT_X * TY;
  __shared__ double sM[HT_K * SZM], sFx[HT_K * SZX], sFy[HT_K * SZY];
  if (!clk->active) return;  // uniform over the block
  const long long N = sc.N;
  const int Nx = sc.Nx, Ny = sc.Ny, Nz = sc.Nz;
  const int tiles_x = (Nx + HT_X - 1) / HT_X, tiles_y = (Ny + TY - 1) / TY;
  const int grp = bid % HT_G;
  int t = bid / HT_G;
  const int tx0 = (t % tiles_x) * HT_X;
  t /= tiles_x;
  const int ty0 = (t % tiles_y) * TY;
  const int k = t / tiles_y;
  const int lx = threadIdx.x % HT_X, ly = threadIdx.x / HT_X;
  const int i = tx0 + lx, j = ty0 + ly;
  const long long plane = (long long)Nx * Ny * k;
  const int n0 = HT_K * grp;
  // stage the group's tiles (clamped coordinates: every load in range)
#pragma unroll 1
  for (int q = 0; q < HT_K; ++q) {
    const long long mo = N * (n0 + q) + plane;
    for (int e = threadIdx.x; e < SZM; e += BS) {
      const int r = e / MX, w = e % MX;
      sM[q * SZM + e] = M[mo + (long long)Nx * min(max(ty0 - 2 + r, 0), Ny - 1) + min(max(tx0 - 2 + w, 0), Nx - 1)];
    }
    for (int e = threadIdx.x; e < SZX; e += BS) {
      const int r = e / MX, w = e % MX;
      sFx[q * SZX + e] = Fx[mo + (long long)Nx * min(ty0 + r, Ny - 1) + min(max(tx0 - 2 + w, 0), Nx - 1)];
    }
    for (int e = threadIdx.x; e < SZY; e += BS) {
      const int r = e / HT_X, w = e % HT_X;
      sFy[q * SZY + e] = Fy[mo + (long long)Nx * min(max(ty0 - 2 + r, 0), Ny - 1) + min(tx0 + w, Nx - 1)];
    }
  }
  __syncthreads();
  if (!(i < Nx && j < Ny)) return;
  const long long c = plane + (long long)Nx * j + i;
  const double dt = clk->dt;
  double acc[HT_K];
  {
    const HllLine X = hll_setup(vp, vp + N, c - i, 1, Nx, i, dt / sc.dx);
    const int colX = int(X.base - (c - i)) - (tx0 - 2);  // cell L of the x line in the tile
#pragma unroll
    for (int q = 0; q < HT_K; ++q) acc[q] = hll_update_at(sM + q * SZM + (ly + 2) * MX + colX, sFx + q * SZX + ly * MX + colX, 1, 1, X);
  }
  {
    const HllLine Y = hll_setup(vp + 2 * N, vp + 3 * N, c - (long long)j * Nx, Nx, Ny, j, dt / sc.dy);
    const int rowY = int((Y.base - (c - (long long)j * Nx)) / Nx) - (ty0 - 2);  // cell L of the y line
#pragma unroll
    for (int q = 0; q < HT_K; ++q)
      acc[q] = acc[q] + hll_update_at(sM + q * SZM + rowY * MX + lx + 2, sFy + q * SZY + rowY * HT_X + lx, MX, HT_X, Y);
  }
  HllLine Z;
  if (Nz > 1) Z = hll_setup(vp + 4 * N, vp + 5 * N, c - (long long)k * Nx * Ny, Nx * Ny, Nz, k, dt / sc.dz);
#pragma unroll
  for (int q = 0; q < HT_K; ++q) {
    const long long mo = N * (n0 + q);
    const double mc = sM[q * SZM + (ly + 2) * MX + lx + 2];
    const double mz = (Nz == 1) ? mc : hll_update(M + mo, Fz + mo, Z);
    Mout[c + mo] = acc[q] + mz - 2.0 * mc;
  }
}

template <int TY, int MINB>
__global__ void __launch_bounds__(HT_X * TY, MINB) k_hll_tile(const double* __restrict__ M, const double* __restrict__ Fx,
                                                         const double* __restrict__ Fy, const double* __restrict__ Fz,
                                                         const double* __restrict__ vp, double* __restrict__ Mout, const StepConst sc,
                                                         const DevClock* clk) {
  hll_tile_body<TY>(M, Fx, Fy, Fz, vp, Mout, sc, clk, blockIdx.x);
}
template <int TY, int MINB>
__global__ void __launch_bounds__(HT_X * TY, MINB) k_hll_tile_b(const Batch bt) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  hll_tile_body<TY>(d.buf[DB_M], d.buf[DB_FX], d.buf[DB_FY], d.buf[DB_FZ], d.buf[DB_VP], d.buf[DB_MTMP], sc, d.clk,
                    blockIdx.x - __ldg(bt.blk0 + m));
}

template <int BS, int GROUPS, int MINB = HQ_MINB_HLL * 256 / BS>
void hll_launch(const double* M, const double* Fx, const double* Fy, const double* Fz, const double* vp, double* Mout, const StepConst& sc,
                const DevClock* clk, cudaStream_t s) {
  k_hll<BS, GROUPS, MINB><<<grid_of(sc.N, BS) * GROUPS, BS, 0, s>>>(M, Fx, Fy, Fz, vp, Mout, sc, clk);
}
void hll_variant(int variant, const double* M, const double* Fx, const double* Fy, const double* Fz, const double* vp, double* Mout,
                 const StepConst& sc, const DevClock* clk, cudaStream_t s) {
  switch (variant) {
    case 1: hll_launch<256, 5>(M, Fx, Fy, Fz, vp, Mout, sc, clk, s); break;
    case 2: hll_launch<256, 7>(M, Fx, Fy, Fz, vp, Mout, sc, clk, s); break;
    case 3: hll_launch<128, 5>(M, Fx, Fy, Fz, vp, Mout, sc, clk, s); break;
    case 4: hll_launch<128, 7>(M, Fx, Fy, Fz, vp, Mout, sc, clk, s); break;
    case 5: hll_launch<128, 1>(M, Fx, Fy, Fz, vp, Mout, sc, clk, s); break;
    case 6: hll_launch<256, 7, 6>(M, Fx, Fy, Fz, vp, Mout, sc, clk, s); break;
    case 7: hll_launch<256, 5, 5>(M, Fx, Fy, Fz, vp, Mout, sc, clk, s); break;
    case 8: k_hll_tile<8, 4><<<hll_blocks(8, sc.Nx, sc.Ny, sc.Nz), HT_X * 8, 0, s>>>(M, Fx, Fy, Fz, vp, Mout, sc, clk); break;
    case 9: k_hll_tile<4, 6><<<hll_blocks(9, sc.Nx, sc.Ny, sc.Nz), HT_X * 4, 0, s>>>(M, Fx, Fy, Fz, vp, Mout, sc, clk); break;
    default: hll_launch<256, 1>(M, Fx, Fy, Fz, vp, Mout, sc, clk, s); break;
  }
}
void hll_variant_b(int variant, const Batch& bt, int nblk, cudaStream_t s) {
  switch (variant) {
    case 1: k_hll_b<256, 5><<<nblk, 256, 0, s>>>(bt); break;
    case 2: k_hll_b<256, 7><<<nblk, 256, 0, s>>>(bt); break;
    case 3: k_hll_b<128, 5><<<nblk, 128, 0, s>>>(bt); break;
    case 4: k_hll_b<128, 7><<<nblk, 128, 0, s>>>(bt); break;
    case 5: k_hll_b<128, 1><<<nblk, 128, 0, s>>>(bt); break;
    case 6: k_hll_b<256, 7, 6><<<nblk, 256, 0, s>>>(bt); break;
    case 7: k_hll_b<256, 5, 5><<<nblk, 256, 0, s>>>(bt); break;
    case 8: k_hll_tile_b<8, 4><<<nblk, HT_X * 8, 0, s>>>(bt); break;
    case 9: k_hll_tile_b<4, 6><<<nblk, HT_X * 4, 0, s>>>(bt); break;
    default: k_hll_b<256, 1><<<nblk, 256, 0, s>>>(bt); break;
  }
}

__global__ void k_set_clock(DevClock* clk, double t, long long nn) {
  clk->t = t; clk->nn = nn; clk->dt = 0.0; clk->vmax = 0.0; clk->active = 0; clk->status = 0;
  for (int q = 0; q < 5; ++q) clk->dense[q] = 0;
  clk->fb_cells = 0; clk->stage_cells = 0;
  for (int q = 0; q < 3; ++q) clk->vdir_bits[q] = 0;
  clk->worst_cell = ~0ull; clk->worst_dir = -1;
  clk->maxdiff = 0.0; clk->maxdiff_nn = -1;
}

// First-step diagnostics (src/simulation_runner.jl:404-470): at step 1 only,
// the largest |speed| along each axis over all cells (Julia `maximum`
// semantics: a NaN wins; |speed| bit patterns order like the values, NaN
// above Inf), then the first cell that attains the global maximum.
__device__ __forceinline__ void diag_speeds_body(const double* __restrict__ vp, const StepConst& sc, DevClock* clk, int bid, int nblk) {
  if (!clk->active || clk->nn != 1) return;
  const long long N = sc.N;
  unsigned long long m[3] = {0, 0, 0};
  for (long long c = (long long)bid * 256 + threadIdx.x; c < N; c += (long long)nblk * 256)
    for (int d = 0; d < 3; ++d)
      for (int q = 0; q < 2; ++q) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(vp[c + N * (2 * d + q)]));
        m[d] = b > m[d] ? b : m[d];
      }
  for (int d = 0; d < 3; ++d) {
    unsigned long long v = m[d];
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
      v = w > v ? w : v;
    }
    if ((threadIdx.x & 31) == 0 && v) atomicMax(&clk->vdir_bits[d], v);
  }
}
__device__ __forceinline__ void diag_worst_body(const double* __restrict__ vp, const StepConst& sc, DevClock* clk, int bid, int nblk) {
  if (!clk->active || clk->nn != 1) return;
  const long long N = sc.N;
  unsigned long long g = clk->vdir_bits[0];
  g = clk->vdir_bits[1] > g ? clk->vdir_bits[1] : g;
  g = clk->vdir_bits[2] > g ? clk->vdir_bits[2] : g;
  for (long long c = (long long)bid * 256 + threadIdx.x; c < N; c += (long long)nblk * 256)
    for (int d = 0; d < 3; ++d)
      for (int q = 0; q < 2; ++q)
        if ((unsigned long long)__double_as_longlong(fabs(vp[c + N * (2 * d + q)])) == g) {
          // lowest cell first, then lowest direction (the reference scans x, y, z)
          const unsigned long long key = ((unsigned long long)c << 2) | (unsigned long long)d;
          atomicMin(&clk->worst_cell, key);
        }
}
__global__ void __launch_bounds__(256) k_diag_speeds(const double* __restrict__ vp, const StepConst sc, DevClock* clk) {
  diag_speeds_body(vp, sc, clk, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(256) k_diag_worst(const double* __restrict__ vp, const StepConst sc, DevClock* clk) {
  diag_worst_body(vp, sc, clk, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(256) k_diag_speeds_b(const Batch bt) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  const int b0 = __ldg(bt.blk0 + m);
  diag_speeds_body(d.buf[DB_VP], sc, d.clk, blockIdx.x - b0, __ldg(bt.blk0 + m + 1) - b0);
}
__global__ void __launch_bounds__(256) k_diag_worst_b(const Batch bt) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  const int b0 = __ldg(bt.blk0 + m);
  diag_worst_body(d.buf[DB_VP], sc, d.clk, blockIdx.x - b0, __ldg(bt.blk0 + m + 1) - b0);
}

// MaxDiff (src/simulation_runner.jl:562-637) of the state after the step, at
// steps nn % interval == 0 and nn == 1: on the diagonal i = j of the first
// z-layer, Diff_m(i) = M_m(i,i) -+ M_m(N'-1-i, N'-1-i) for the moments
// M000, M100, M200, M300, M400 (- for the even ones, + for the odd ones),
// MaxDiff = max_m |max_i Diff_m(i) / (||Diff_m||_2 + 1)|; NaN propagates.
__device__ __forceinline__ void maxdiff_body(const double* __restrict__ M, const StepConst& sc, DevClock* clk) {
  if (!clk->active || sc.symmetry_check_interval <= 0) return;
  const long long nn = clk->nn;
  if (!(nn % sc.symmetry_check_interval == 0 || nn == 1)) return;
  const int Nd = sc.Nx < sc.Ny ? sc.Nx : sc.Ny;
  const long long N = sc.N;
  __shared__ double smax[5][8], ssq[5][8];
  double mx[5], sq[5];
  for (int m = 0; m < 5; ++m) { mx[m] = -INFINITY; sq[m] = 0.0; }
  for (int i = threadIdx.x; i < Nd; i += 256) {
    const int j = Nd - 1 - i;
    const long long a = (long long)i + (long long)sc.Nx * i, b = (long long)j + (long long)sc.Nx * j;
    for (int m = 0; m < 5; ++m) {
      const double d = (m & 1) ? M[a + N * m] + M[b + N * m] : M[a + N * m] - M[b + N * m];
      mx[m] = nanmax(mx[m], d);
      sq[m] = sq[m] + d * d;
    }
  }
  for (int m = 0; m < 5; ++m) {
    mx[m] = warp_nanmax(mx[m]);
    double v = sq[m];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) { smax[m][threadIdx.x >> 5] = mx[m]; ssq[m][threadIdx.x >> 5] = v; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double md = 0.0;
    for (int m = 0; m < 5; ++m) {
      double a = -INFINITY, q = 0.0;
      for (int w = 0; w < 8; ++w) { a = nanmax(a, smax[m][w]); q = q + ssq[m][w]; }
      md = nanmax(md, fabs(a / (sqrt(q) + 1.0)));
    }
    clk->maxdiff = md;
    clk->maxdiff_nn = nn;
  }
}


__global__ void __launch_bounds__(256) k_maxdiff(const double* __restrict__ M, const StepConst sc, DevClock* clk) { maxdiff_body(M, sc, clk); }
// fused batch: one block per member
__global__ void __launch_bounds__(256) k_maxdiff_b(const Batch bt) {
  const Dom& d = bt.dom[blockIdx.x];
  const StepConst sc = d.sc;
  maxdiff_body(d.buf[DB_M], sc, d.clk);
}

}  // namespace

// ------------------------------------------------------------------ C-ABI
struct hyq_ctx {
  hyq_params p;
  StepConst sc;
  long long N;
  int device;
  double *M = nullptr, *Mtmp = nullptr, *Fx = nullptr, *Fy = nullptr, *Fz = nullptr, *vp = nullptr, *blockmax = nullptr;
  DevClock* clk = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // the step split at the CFL reduction (hyq_step_begin / hyq_step_end),
  // captured on first use; xchg: the local / global max |speed| and NaN flag
  cudaGraphExec_t exec_a = nullptr, exec_b = nullptr;
  double* xchg = nullptr;
  // hyq_step_host: copy stream and per-slab events, made on first use
  cudaStream_t cstream = nullptr;
  std::vector<cudaEvent_t> up, down;
  // learned mode: the network's seeds [6][N], its weight image and error word
  float* seeds = nullptr;
  WaveNet net{nullptr, nullptr};
  float* net_w = nullptr;  // FP32 parameters (device), packed into net.image
  bool net_loaded = false;
  // launch shape of the HLL kernel (hll_shape; hyq_set_variant)
  int hll_variant = 0;
  // bumped whenever the step graph is captured again (a batch holding this
  // member re-reads its constants then)
  int gen = 0;
  std::string err;
};

namespace {
thread_local std::string g_err;

int fail(hyq_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg; else g_err = msg;
  return code;
}
int cuda_fail(hyq_ctx* ctx, cudaError_t e, const char* what) {
  return fail(ctx, HYQ_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define HQ_CHECK(ctx, call)                                       \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);    \
  } while (0)


void enqueue_step(hyq_ctx* ctx, cudaStream_t s) {
  launch_phase_A(ctx->sc, ctx->M, ctx->Mtmp, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->blockmax, ctx->clk, s, nullptr, 0, -1, &ctx->net);
  k_cfl<<<1, 1024, 0, s>>>(ctx->blockmax, ctx->sc, ctx->clk);
  launch_diagnostics_speeds(ctx->vp, ctx->sc, ctx->clk, s);
  hll_variant(ctx->hll_variant, ctx->M, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->Mtmp, ctx->sc, ctx->clk, s);
  launch_phase_EF(ctx->sc, ctx->Mtmp, ctx->M, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->clk, s);
  launch_maxdiff(ctx->M, ctx->sc, ctx->clk, s);
}
// Capture one step as the context's graph (replacing an earlier one).
int capture_graph(hyq_ctx* ctx) {
  cudaError_t e;
  ++ctx->gen;
  if (ctx->exec) { cudaGraphExecDestroy(ctx->exec); ctx->exec = nullptr; }
  if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
  if ((e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return cuda_fail(ctx, e, "cudaStreamBeginCapture");
  enqueue_step(ctx, ctx->stream);
  if ((e = cudaStreamEndCapture(ctx->stream, &ctx->graph)) != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
  if ((e = cudaGraphInstantiate(&ctx->exec, ctx->graph, 0)) != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
  return HYQ_OK;
}

// The two halves of a step around the CFL reduction, each as a graph.
void enqueue_half_a(hyq_ctx* ctx, cudaStream_t s) {
  launch_phase_A(ctx->sc, ctx->M, ctx->Mtmp, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->blockmax, ctx->clk, s, nullptr, 0, -1, &ctx->net);
  k_vmax_local<<<1, 1024, 0, s>>>(ctx->blockmax, ctx->sc, ctx->clk, ctx->xchg);
}
void enqueue_half_b(hyq_ctx* ctx, cudaStream_t s) {
  k_cfl_global<<<1, 1, 0, s>>>(ctx->xchg, ctx->sc, ctx->clk);
  launch_diagnostics_speeds(ctx->vp, ctx->sc, ctx->clk, s);
  hll_variant(ctx->hll_variant, ctx->M, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->Mtmp, ctx->sc, ctx->clk, s);
  launch_phase_EF(ctx->sc, ctx->Mtmp, ctx->M, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->clk, s);
  launch_maxdiff(ctx->M, ctx->sc, ctx->clk, s);
}
int capture_one(hyq_ctx* ctx, void (*fn)(hyq_ctx*, cudaStream_t), cudaGraphExec_t* exec) {
  cudaError_t e;
  cudaGraph_t g = nullptr;
  if (*exec) { cudaGraphExecDestroy(*exec); *exec = nullptr; }
  if ((e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamBeginCapture");
  fn(ctx, ctx->stream);
  if ((e = cudaStreamEndCapture(ctx->stream, &g)) != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
  return HYQ_OK;
}
int capture_halves(hyq_ctx* ctx) {
  if (!ctx->xchg) HQ_CHECK(ctx, cudaMalloc((void**)&ctx->xchg, 2 * sizeof(double)));
  int r = capture_one(ctx, enqueue_half_a, &ctx->exec_a);
  if (r == HYQ_OK) r = capture_one(ctx, enqueue_half_b, &ctx->exec_b);
  return r;
}

int net_status(hyq_ctx* ctx) {
  if (ctx->sc.mode != MODE_LEARNED) return HYQ_OK;
  int h = 0;
  HQ_CHECK(ctx, cudaMemcpyAsync(&h, ctx->net.err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  if (h) return fail(ctx, HYQ_ETIMEOUT, "the wave-speed network kernel gave up waiting for its tensor-core operations");
  return HYQ_OK;
}

__global__ void k_reset_counters(DevClock* clk) { clk->fb_cells = 0; clk->stage_cells = 0; }
// The device IC fill (hyq_set_state_ic): one thread per cell, the regions
// and moments in constant-size parameter arrays read through global memory.
constexpr int IC_MAX_REGIONS = 64;
__global__ void __launch_bounds__(256) k_fill_ic(double* __restrict__ M, const StepConst sc, const double* __restrict__ xyz, double dx,
                                                 double dy, double dz, const double* __restrict__ bg, int nreg,
                                                 const hyq_ic_region* __restrict__ regs, const double* __restrict__ mom) {
  const long long N = sc.N;
  const long long c = (long long)blockIdx.x * 256 + threadIdx.x;
  if (c >= N) return;
  const int i = int(c % sc.Nx), j = int((c / sc.Nx) % sc.Ny), k = int(c / ((long long)sc.Nx * sc.Ny));
  const double x = xyz[i], y = xyz[sc.Nx + j], z = xyz[sc.Nx + sc.Ny + k];
  int use = -1;
  for (int r = 0; r < nreg; ++r) {
    const hyq_ic_region& g = regs[r];
    bool in;
    if (g.kind == 1) {
      in = i >= g.i0 && i <= g.i1 && j >= g.j0 && j <= g.j1 && k >= g.k0 && k <= g.k1;
    } else if (g.everywhere) {
      in = true;
    } else {
      in = jmax(x - dx / 2.0, g.lo[0]) < jmin(x + dx / 2.0, g.hi[0]) && jmax(y - dy / 2.0, g.lo[1]) < jmin(y + dy / 2.0, g.hi[1]) &&
           jmax(z - dz / 2.0, g.lo[2]) < jmin(z + dz / 2.0, g.hi[2]);
    }
    if (in) use = r;
  }
  const double* src = use < 0 ? bg : mom + 35 * use;
#pragma unroll
  for (int n = 0; n < 35; ++n) M[c + N * n] = src[n];
}
}  // namespace

// Launch helpers for other translation units (same kernels and shapes as
// enqueue_step).
namespace hyqk {
void launch_cfl(const double* blockmax, const StepConst& sc, DevClock* clk, cudaStream_t s) {
  k_cfl<<<1, 1024, 0, s>>>(blockmax, sc, clk);
}
void launch_hll(const double* M, const double* Fx, const double* Fy, const double* Fz, const double* vp, double* Mout, const StepConst& sc,
                const DevClock* clk, cudaStream_t s, int variant) {
  hll_variant(variant, M, Fx, Fy, Fz, vp, Mout, sc, clk, s);
}
void launch_set_clock(DevClock* clk, double t, long long nn, cudaStream_t s) { k_set_clock<<<1, 1, 0, s>>>(clk, t, nn); }
void launch_diagnostics_speeds(const double* vp, const StepConst& sc, DevClock* clk, cudaStream_t s) {
  const int g = (int)((sc.N + 255) / 256 < 148 * 8 ? (sc.N + 255) / 256 : 148 * 8);
  k_diag_speeds<<<g, 256, 0, s>>>(vp, sc, clk);
  k_diag_worst<<<g, 256, 0, s>>>(vp, sc, clk);
}
void launch_maxdiff(const double* M, const StepConst& sc, DevClock* clk, cudaStream_t s) { k_maxdiff<<<1, 256, 0, s>>>(M, sc, clk); }
void launch_mid_batch(const BatchPlan& bp, cudaStream_t s) {
  k_cfl_b<<<bp.n, 1024, 0, s>>>(bp.of(DK_ONE));
  k_diag_speeds_b<<<bp.nblk[DK_DIAG], 256, 0, s>>>(bp.of(DK_DIAG));
  k_diag_worst_b<<<bp.nblk[DK_DIAG], 256, 0, s>>>(bp.of(DK_DIAG));
  hll_variant_b(bp.hll_variant, bp.of(DK_HLL), bp.nblk[DK_HLL], s);
}
void launch_maxdiff_batch(const BatchPlan& bp, cudaStream_t s) { k_maxdiff_b<<<bp.n, 256, 0, s>>>(bp.of(DK_ONE)); }
int report_error(int code, const char* msg) { return fail(nullptr, code, msg); }
}  // namespace hyqk

extern "C" {

int hyq_abi_version(void) { return HYQ_ABI_VERSION; }

const char* hyq_last_error(const hyq_ctx* ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

int hyq_create(const hyq_params* p, hyq_ctx** out) {
  if (!p || !out) return fail(nullptr, HYQ_EINVAL, "null argument");
  *out = nullptr;
  if (p->Nx < 2 || p->Ny < 2 || p->Nz < 1)
    return fail(nullptr, HYQ_EINVAL, "grid must have Nx >= 2, Ny >= 2, Nz >= 1 (pas_HLL needs two cells per row)");
  if (!(p->CFL > 0) || !(p->Kn > 0) || !(p->dtmax > 0))
    return fail(nullptr, HYQ_EINVAL, "CFL, Kn and dtmax must be positive");
  if ((long long)p->Nx * p->Ny * p->Nz >= (1LL << 29))
    return fail(nullptr, HYQ_EINVAL, "grid must have fewer than 2^29 cells (the step's cell lists hold 32-bit entries)");
  if (p->mode != HYQ_MODE_PLAIN && p->mode != HYQ_MODE_LEARNED && p->mode != HYQ_MODE_CERTIFIED)
    return fail(nullptr, HYQ_EINVAL, "mode must be HYQ_MODE_PLAIN, HYQ_MODE_LEARNED or HYQ_MODE_CERTIFIED");
  hyq_ctx* ctx = new hyq_ctx();
  ctx->p = *p;
  ctx->device = p->device;
  cudaError_t e = cudaSetDevice(p->device);
  if (e != cudaSuccess) { int r = cuda_fail(nullptr, e, "cudaSetDevice"); delete ctx; return r; }
  const long long N = (long long)p->Nx * p->Ny * p->Nz;
  ctx->N = N;
  StepConst& sc = ctx->sc;
  sc.N = N; sc.Nx = p->Nx; sc.Ny = p->Ny; sc.Nz = p->Nz; sc.flag2D = p->flag2D; sc.positivity = p->positivity;
  sc.nnmax = p->nnmax; sc.tmax = p->tmax; sc.Kn = p->Kn; sc.Ma = p->Ma; sc.CFL = p->CFL; sc.dtmax = p->dtmax;
  sc.dx = (p->xmax - p->xmin) / p->Nx; sc.dy = (p->ymax - p->ymin) / p->Ny; sc.dz = (p->zmax - p->zmin) / p->Nz;
  sc.nblocksA = grid_of(N, BS_A);
  sc.mode = p->mode;
  sc.symmetry_check_interval = p->symmetry_check_interval;
  sc.seeds = nullptr;
  sc.seed_margin = 0.0;
  const size_t b35 = sizeof(double) * 35 * (size_t)N;
  auto alloc = [&](double** ptr, size_t bytes) { return cudaMalloc((void**)ptr, bytes); };
  if (alloc(&ctx->M, b35) != cudaSuccess || alloc(&ctx->Mtmp, b35) != cudaSuccess || alloc(&ctx->Fx, b35) != cudaSuccess ||
      alloc(&ctx->Fy, b35) != cudaSuccess || alloc(&ctx->Fz, b35) != cudaSuccess ||
      alloc(&ctx->vp, sizeof(double) * (7 * (size_t)N + 16)) != cudaSuccess ||
      alloc(&ctx->blockmax, sizeof(double) * (size_t)sc.nblocksA) != cudaSuccess ||
      cudaMalloc((void**)&ctx->clk, sizeof(DevClock)) != cudaSuccess) {
    cudaGetLastError();
    hyq_destroy(ctx);
    return fail(nullptr, HYQ_ENOMEM, "device allocation failed");
  }
  if (p->mode == HYQ_MODE_LEARNED) {
    if (cudaMalloc((void**)&ctx->seeds, sizeof(float) * 6 * (size_t)N) != cudaSuccess ||
        cudaMalloc((void**)&ctx->net.image, (size_t)hyq_net_image_bytes()) != cudaSuccess ||
        cudaMalloc((void**)&ctx->net.err, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&ctx->net_w, sizeof(float) * HYQ_NET_PARAMS) != cudaSuccess) {
      cudaGetLastError();
      hyq_destroy(ctx);
      return fail(nullptr, HYQ_ENOMEM, "device allocation failed");
    }
    if ((e = net_set_smem()) != cudaSuccess || (e = cudaMemset(ctx->net.err, 0, sizeof(int))) != cudaSuccess) {
      int r = cuda_fail(nullptr, e, "network set-up");
      hyq_destroy(ctx);
      return r;
    }
    sc.seeds = ctx->seeds;
  }
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    int r = cuda_fail(nullptr, e, "cudaStreamCreate");
    hyq_destroy(ctx);
    return r;
  }
  k_set_clock<<<1, 1, 0, ctx->stream>>>(ctx->clk, 0.0, 0);
  // capture one step as a graph
  if (capture_graph(ctx) != HYQ_OK) {
    const std::string msg = ctx->err;
    hyq_destroy(ctx);
    return fail(nullptr, HYQ_ECUDA, msg);
  }
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
    int r = cuda_fail(nullptr, e, "create sync"); hyq_destroy(ctx); return r;
  }
  *out = ctx;
  return HYQ_OK;
}

void hyq_destroy(hyq_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->exec) cudaGraphExecDestroy(ctx->exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  if (ctx->exec_a) cudaGraphExecDestroy(ctx->exec_a);
  if (ctx->exec_b) cudaGraphExecDestroy(ctx->exec_b);
  if (ctx->xchg) cudaFree(ctx->xchg);
  double* bufs[] = {ctx->M, ctx->Mtmp, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->blockmax};
  for (double* b : bufs) if (b) cudaFree(b);
  if (ctx->clk) cudaFree(ctx->clk);
  if (ctx->seeds) cudaFree(ctx->seeds);
  if (ctx->net.image) cudaFree(ctx->net.image);
  if (ctx->net.err) cudaFree(ctx->net.err);
  if (ctx->net_w) cudaFree(ctx->net_w);
  if (ctx->cstream) cudaStreamSynchronize(ctx->cstream);
  for (cudaEvent_t e : ctx->up) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->down) cudaEventDestroy(e);
  if (ctx->cstream) cudaStreamDestroy(ctx->cstream);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

void* hyq_stream(hyq_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int hyq_set_clock(hyq_ctx* ctx, double t, int64_t nn) {
  if (!ctx) return fail(nullptr, HYQ_EINVAL, "null ctx");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  k_set_clock<<<1, 1, 0, ctx->stream>>>(ctx->clk, t, (long long)nn);
  HQ_CHECK(ctx, cudaGetLastError());
  return HYQ_OK;
}

int hyq_set_state(hyq_ctx* ctx, const double* M) {
  if (!ctx || !M) return fail(ctx, HYQ_EINVAL, "null argument");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaMemcpyAsync(ctx->M, M, sizeof(double) * 35 * ctx->N, cudaMemcpyHostToDevice, ctx->stream));
  k_set_clock<<<1, 1, 0, ctx->stream>>>(ctx->clk, 0.0, 0);
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  return HYQ_OK;
}

int hyq_set_state_ic(hyq_ctx* ctx, const double* xm, const double* ym, const double* zm, double dx, double dy, double dz,
                     const double* bg, int32_t nregions, const hyq_ic_region* regions, const double* moments) {
  if (!ctx || !xm || !ym || !zm || !bg || nregions < 0 || (nregions > 0 && (!regions || !moments)))
    return fail(ctx, HYQ_EINVAL, "null argument");
  if (nregions > IC_MAX_REGIONS) return fail(ctx, HYQ_EINVAL, "at most 64 regions");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  // one small upload of the tables: centres, background, regions, moments
  const int nx = ctx->p.Nx, ny = ctx->p.Ny, nz = ctx->p.Nz;
  std::vector<double> tab((size_t)nx + ny + nz + 35 + 35 * (size_t)nregions);
  std::memcpy(tab.data(), xm, sizeof(double) * nx);
  std::memcpy(tab.data() + nx, ym, sizeof(double) * ny);
  std::memcpy(tab.data() + nx + ny, zm, sizeof(double) * nz);
  std::memcpy(tab.data() + nx + ny + nz, bg, sizeof(double) * 35);
  if (nregions) std::memcpy(tab.data() + nx + ny + nz + 35, moments, sizeof(double) * 35 * nregions);
  // the tables ride in the flux buffer Fx (dead between steps)
  const size_t rbytes = sizeof(hyq_ic_region) * (size_t)nregions;
  double* dtab = ctx->Fx;
  hyq_ic_region* dreg = reinterpret_cast<hyq_ic_region*>(ctx->Fx + tab.size() + 8);
  if ((tab.size() + 8) * sizeof(double) + rbytes > sizeof(double) * 35 * (size_t)ctx->N)
    return fail(ctx, HYQ_EINVAL, "grid too small for the IC tables");
  HQ_CHECK(ctx, cudaMemcpyAsync(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, ctx->stream));
  if (nregions) HQ_CHECK(ctx, cudaMemcpyAsync(dreg, regions, rbytes, cudaMemcpyHostToDevice, ctx->stream));
  k_fill_ic<<<grid_of(ctx->N, 256), 256, 0, ctx->stream>>>(ctx->M, ctx->sc, dtab, dx, dy, dz, dtab + nx + ny + nz, nregions, dreg,
                                                           dtab + nx + ny + nz + 35);
  k_set_clock<<<1, 1, 0, ctx->stream>>>(ctx->clk, 0.0, 0);
  HQ_CHECK(ctx, cudaGetLastError());
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  return HYQ_OK;
}

int hyq_set_state_device(hyq_ctx* ctx, const double* dM) {
  if (!ctx || !dM) return fail(ctx, HYQ_EINVAL, "null argument");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaMemcpyAsync(ctx->M, dM, sizeof(double) * 35 * ctx->N, cudaMemcpyDeviceToDevice, ctx->stream));
  k_set_clock<<<1, 1, 0, ctx->stream>>>(ctx->clk, 0.0, 0);
  HQ_CHECK(ctx, cudaGetLastError());
  return HYQ_OK;
}

int hyq_get_state(hyq_ctx* ctx, double* M) {
  if (!ctx || !M) return fail(ctx, HYQ_EINVAL, "null argument");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaMemcpyAsync(M, ctx->M, sizeof(double) * 35 * ctx->N, cudaMemcpyDeviceToHost, ctx->stream));
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  return HYQ_OK;
}

int hyq_get_state_device(hyq_ctx* ctx, double* dM) {
  if (!ctx || !dM) return fail(ctx, HYQ_EINVAL, "null argument");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaMemcpyAsync(dM, ctx->M, sizeof(double) * 35 * ctx->N, cudaMemcpyDeviceToDevice, ctx->stream));
  return HYQ_OK;
}

int hyq_reset_counters(hyq_ctx* ctx) {
  if (!ctx) return fail(nullptr, HYQ_EINVAL, "null ctx");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  k_reset_counters<<<1, 1, 0, ctx->stream>>>(ctx->clk);
  HQ_CHECK(ctx, cudaGetLastError());
  return HYQ_OK;
}

int hyq_set_wavespeed_net(hyq_ctx* ctx, const float* w, double margin) {
  if (!ctx || !w) return fail(ctx, HYQ_EINVAL, "null argument");
  if (ctx->sc.mode != MODE_LEARNED) return fail(ctx, HYQ_EINVAL, "the context was not created with HYQ_MODE_LEARNED");
  if (!(margin >= 0.0) || !(margin < 8.0)) return fail(ctx, HYQ_EINVAL, "margin must be in [0, 8)");
  for (int i = 0; i < HYQ_NET_PARAMS; ++i)
    if (!std::isfinite(w[i])) return fail(ctx, HYQ_EINVAL, "network parameters must be finite");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaMemcpyAsync(ctx->net_w, w, sizeof(float) * HYQ_NET_PARAMS, cudaMemcpyHostToDevice, ctx->stream));
  int r = hyq_net_pack(ctx->net_w, ctx->net.image, ctx->stream);
  if (r != HYQ_OK) return fail(ctx, r, hyq_last_error(nullptr));
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->sc.seed_margin = margin;
  // the margin is a kernel argument of the captured step
  if ((r = capture_graph(ctx)) != HYQ_OK) return r;
  if (ctx->exec_a && (r = capture_halves(ctx)) != HYQ_OK) return r;
  ctx->net_loaded = true;
  return HYQ_OK;
}

int hyq_set_spacing(hyq_ctx* ctx, double dx, double dy, double dz) {
  if (!ctx) return fail(nullptr, HYQ_EINVAL, "null ctx");
  if (!(dx > 0) || !(dy > 0) || !(dz > 0)) return fail(ctx, HYQ_EINVAL, "spacings must be positive");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->sc.dx = dx; ctx->sc.dy = dy; ctx->sc.dz = dz;
  int r = capture_graph(ctx);
  if (r == HYQ_OK && ctx->exec_a) r = capture_halves(ctx);
  return r;
}

int32_t hyq_variant_count(int32_t kernel) {
  if (kernel == HYQ_KERNEL_HLL) return HLL_VARIANTS;
  if (kernel == HYQ_KERNEL_CORR) return HYQ_CORR_VARIANTS;
  return 0;
}

int hyq_set_variant(hyq_ctx* ctx, int32_t kernel, int32_t variant) {
  if (!ctx) return fail(nullptr, HYQ_EINVAL, "null ctx");
  if (kernel != HYQ_KERNEL_HLL) return fail(ctx, HYQ_EINVAL, "a context has launch variants for HYQ_KERNEL_HLL only");
  if (variant < 0 || variant >= HLL_VARIANTS) return fail(ctx, HYQ_EINVAL, "variant out of range");
  if (variant == ctx->hll_variant) return HYQ_OK;
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->hll_variant = variant;
  int r = capture_graph(ctx);
  if (r == HYQ_OK && ctx->exec_a) r = capture_halves(ctx);
  return r;
}

int hyq_step_begin(hyq_ctx* ctx, double* xchg) {
  if (!ctx || !xchg) return fail(ctx, HYQ_EINVAL, "null argument");
  if (ctx->sc.mode == MODE_LEARNED && !ctx->net_loaded)
    return fail(ctx, HYQ_EINVAL, "HYQ_MODE_LEARNED needs the wave-speed network (hyq_set_wavespeed_net) before stepping");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  if (!ctx->exec_a) {
    const int r = capture_halves(ctx);
    if (r != HYQ_OK) return r;
  }
  HQ_CHECK(ctx, cudaGraphLaunch(ctx->exec_a, ctx->stream));
  HQ_CHECK(ctx, cudaMemcpyAsync(xchg, ctx->xchg, 2 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  return HYQ_OK;
}

int hyq_step_end(hyq_ctx* ctx, const double* xchg) {
  if (!ctx || !xchg) return fail(ctx, HYQ_EINVAL, "null argument");
  if (!ctx->exec_b) return fail(ctx, HYQ_EINVAL, "hyq_step_end without hyq_step_begin");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaMemcpyAsync(ctx->xchg, xchg, 2 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  HQ_CHECK(ctx, cudaGraphLaunch(ctx->exec_b, ctx->stream));
  return HYQ_OK;
}

int hyq_copy_layers(hyq_ctx* ctx, int32_t k0, int32_t nk, double* buf, int32_t into_state) {
  if (!ctx || !buf || nk < 0 || k0 < 0 || k0 + nk > ctx->p.Nz) return fail(ctx, HYQ_EINVAL, "bad layer range");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  const size_t layer = (size_t)ctx->p.Nx * ctx->p.Ny;
  const size_t w = sizeof(double) * layer * (size_t)nk, pitch_state = sizeof(double) * (size_t)ctx->N;
  double* st = ctx->M + layer * (size_t)k0;
  if (into_state)
    HQ_CHECK(ctx, cudaMemcpy2DAsync(st, pitch_state, buf, w, w, 35, cudaMemcpyDeviceToDevice, ctx->stream));
  else
    HQ_CHECK(ctx, cudaMemcpy2DAsync(buf, w, st, pitch_state, w, 35, cudaMemcpyDeviceToDevice, ctx->stream));
  return HYQ_OK;
}

int hyq_advance_async(hyq_ctx* ctx, int64_t max_steps) {
  if (!ctx || max_steps < 0) return fail(ctx, HYQ_EINVAL, "bad argument");
  if (ctx->sc.mode == MODE_LEARNED && !ctx->net_loaded)
    return fail(ctx, HYQ_EINVAL, "HYQ_MODE_LEARNED needs the wave-speed network (hyq_set_wavespeed_net) before stepping");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  for (int64_t s = 0; s < max_steps; ++s) HQ_CHECK(ctx, cudaGraphLaunch(ctx->exec, ctx->stream));
  return HYQ_OK;
}

int hyq_advance_timed(hyq_ctx* ctx, int64_t steps, float* ms) {
  if (!ctx || !ms || steps < 0) return fail(ctx, HYQ_EINVAL, "bad argument");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  constexpr int K = HYQ_TIMED_SLOTS;
  cudaEvent_t ev[K + 1];
  for (int q = 0; q <= K; ++q) HQ_CHECK(ctx, cudaEventCreate(&ev[q]));
  for (int q = 0; q < K; ++q) ms[q] = 0.0f;
  cudaStream_t s = ctx->stream;
  for (int64_t it = 0; it < steps; ++it) {
    cudaEventRecord(ev[0], s);
    launch_phase_A(ctx->sc, ctx->M, ctx->Mtmp, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->blockmax, ctx->clk, s, ev + 1, 0, -1, &ctx->net);
    k_cfl<<<1, 1024, 0, s>>>(ctx->blockmax, ctx->sc, ctx->clk);
    launch_diagnostics_speeds(ctx->vp, ctx->sc, ctx->clk, s);
    cudaEventRecord(ev[6], s);
    hll_variant(ctx->hll_variant, ctx->M, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->Mtmp, ctx->sc, ctx->clk, s);
    cudaEventRecord(ev[7], s);
    launch_phase_EF(ctx->sc, ctx->Mtmp, ctx->M, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->clk, s, ev + 8);
    launch_maxdiff(ctx->M, ctx->sc, ctx->clk, s);
    HQ_CHECK(ctx, cudaEventSynchronize(ev[K]));
    for (int q = 0; q < K; ++q) {
      float t = 0.0f;
      cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
      ms[q] += t;
    }
  }
  for (int q = 0; q <= K; ++q) cudaEventDestroy(ev[q]);
  HQ_CHECK(ctx, cudaGetLastError());
  return HYQ_OK;
}

int hyq_synchronize(hyq_ctx* ctx) {
  if (!ctx) return fail(nullptr, HYQ_EINVAL, "null ctx");
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  return HYQ_OK;
}

int hyq_stats_get(hyq_ctx* ctx, hyq_stats* out) {
  if (!ctx || !out) return fail(ctx, HYQ_EINVAL, "null argument");
  DevClock h;
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  HQ_CHECK(ctx, cudaMemcpyAsync(&h, ctx->clk, sizeof(DevClock), cudaMemcpyDeviceToHost, ctx->stream));
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  out->t = h.t; out->dt = h.dt; out->vmax = h.vmax; out->nn = h.nn; out->status = h.status;
  out->done = (h.t < ctx->p.tmax && h.nn < ctx->p.nnmax) ? 0 : 1;
  out->stage_cells = (int64_t)h.stage_cells;
  out->fallback_cells = (int64_t)h.fb_cells;
  out->dense_mask = 0;
  for (int q = 0; q < 5; ++q) out->dense_mask |= (h.dense[q] > 0 ? 1 : 0) << q;
  for (int q = 0; q < 3; ++q) {
    double v;
    std::memcpy(&v, &h.vdir_bits[q], sizeof v);
    out->vmax_first[q] = v;
  }
  out->worst_cell = h.worst_cell == ~0ull ? -1 : (int64_t)(h.worst_cell >> 2);
  out->worst_dir = h.worst_cell == ~0ull ? -1 : (int32_t)(h.worst_cell & 3ull);
  out->maxdiff = h.maxdiff;
  out->maxdiff_step = h.maxdiff_nn;
  return HYQ_OK;
}

int hyq_advance(hyq_ctx* ctx, int64_t max_steps, double* t, int64_t* nn, int32_t* done) {
  int r = hyq_advance_async(ctx, max_steps);
  if (r) return r;
  if ((r = net_status(ctx)) != HYQ_OK) return r;
  hyq_stats st;
  r = hyq_stats_get(ctx, &st);
  if (r) return r;
  if (t) *t = st.t;
  if (nn) *nn = st.nn;
  if (done) *done = st.done;
  if (st.status > 0)
    return fail(ctx, HYQ_ENONFINITE,
                "non-finite CFL wave speed at step " + std::to_string(st.status) +
                    " (a flux Jacobian with Inf/NaN entries; the reference's eigvals throws there)");
  return HYQ_OK;
}

namespace {
constexpr double STEP_HOST_RATIO_A = 1.6, STEP_HOST_RATIO_EF = 0.8;
// Slab boundaries (cells) of S slabs of whole BS_A-cell blocks, slab k's share
// of the nblk blocks in proportion to ratio^k, at least one block each.  The
// share of slabs 0..k-1 is the geometric sum's fraction, written so that no
// power overflows however many slabs are asked for.
void slab_cuts(long long N, long long nblk, int S, double ratio, std::vector<long long>& cut) {
  cut.assign(S + 1, 0);
  auto frac = [&](int k) {
    if (ratio == 1.0) return (double)k / S;
    if (ratio > 1.0) {
      const double a = pow(ratio, (double)(k - S)), b = pow(ratio, (double)-S);
      return (a - b) / (1.0 - b);
    }
    return (1.0 - pow(ratio, (double)k)) / (1.0 - pow(ratio, (double)S));
  };
  long long prev = 0;
  for (int k = 1; k < S; ++k) {
    long long b = (long long)llround((double)nblk * frac(k));
    b = std::max(b, prev + 1);
    b = std::min(b, nblk - (S - k));
    cut[k] = b * BS_A;
    prev = b;
  }
  cut[S] = N;
}
}  // namespace

int hyq_step_host(hyq_ctx* ctx, const double* M_in, double* M_out, int32_t nslabs, double* t, int64_t* nn, int32_t* done) {
  if (!ctx || !M_in || !M_out || nslabs < 1) return fail(ctx, HYQ_EINVAL, "bad argument");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  const long long N = ctx->N;
  // slabs of whole 128-cell blocks (the per-block CFL maxima stay aligned)
  const long long nblk = (N + BS_A - 1) / BS_A;
  const int S = (int)((nslabs < nblk) ? nslabs : nblk);
  if (!ctx->cstream) HQ_CHECK(ctx, cudaStreamCreateWithFlags(&ctx->cstream, cudaStreamNonBlocking));
  while ((int)ctx->up.size() < S) {
    cudaEvent_t a, b;
    HQ_CHECK(ctx, cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    HQ_CHECK(ctx, cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    ctx->up.push_back(a);
    ctx->down.push_back(b);
  }
  // Only the first upload and the last download are not hidden under
  // compute, so the slabs are unequal: phase A's grow by STEP_HOST_RATIO_A
  // (the next slab uploads while phase A runs on this one, and phase A costs
  // about twice the upload), phases E+F's shrink by STEP_HOST_RATIO_EF.
  std::vector<long long> cut, cute;
  slab_cuts(N, nblk, S, STEP_HOST_RATIO_A, cut);
  slab_cuts(N, nblk, S, STEP_HOST_RATIO_EF, cute);
  const size_t pitch = sizeof(double) * (size_t)N;
  cudaStream_t s = ctx->stream, cs = ctx->cstream;
  // upload slab k, then phase A on slab k while slab k+1 is uploading
  for (int k = 0; k < S; ++k) {
    const long long c0 = cut[k], c1 = cut[k + 1];
    HQ_CHECK(ctx, cudaMemcpy2DAsync(ctx->M + c0, pitch, M_in + c0, pitch, sizeof(double) * (size_t)(c1 - c0), 35, cudaMemcpyHostToDevice, cs));
    HQ_CHECK(ctx, cudaEventRecord(ctx->up[k], cs));
    HQ_CHECK(ctx, cudaStreamWaitEvent(s, ctx->up[k], 0));
    launch_phase_A(ctx->sc, ctx->M, ctx->Mtmp, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->blockmax, ctx->clk, s, nullptr, c0, c1, &ctx->net);
  }
  // the CFL reduction and the HLL sweep need every cell
  k_cfl<<<1, 1024, 0, s>>>(ctx->blockmax, ctx->sc, ctx->clk);
  launch_diagnostics_speeds(ctx->vp, ctx->sc, ctx->clk, s);
  hll_variant(ctx->hll_variant, ctx->M, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->Mtmp, ctx->sc, ctx->clk, s);
  // phases E+F slab by slab, each slab downloaded as soon as it is done
  for (int k = 0; k < S; ++k) {
    const long long c0 = cute[k], c1 = cute[k + 1];
    launch_phase_EF(ctx->sc, ctx->Mtmp, ctx->M, ctx->Fx, ctx->Fy, ctx->Fz, ctx->vp, ctx->clk, s, nullptr, c0, c1);
    HQ_CHECK(ctx, cudaEventRecord(ctx->down[k], s));
    HQ_CHECK(ctx, cudaStreamWaitEvent(cs, ctx->down[k], 0));
    HQ_CHECK(ctx, cudaMemcpy2DAsync(M_out + c0, pitch, ctx->M + c0, pitch, sizeof(double) * (size_t)(c1 - c0), 35, cudaMemcpyDeviceToHost, cs));
  }
  launch_maxdiff(ctx->M, ctx->sc, ctx->clk, s);
  HQ_CHECK(ctx, cudaGetLastError());
  HQ_CHECK(ctx, cudaStreamSynchronize(cs));
  hyq_stats st;
  const int r = hyq_stats_get(ctx, &st);
  if (r) return r;
  if (t) *t = st.t;
  if (nn) *nn = st.nn;
  if (done) *done = st.done;
  if (st.status > 0)
    return fail(ctx, HYQ_ENONFINITE,
                "non-finite CFL wave speed at step " + std::to_string(st.status) +
                    " (a flux Jacobian with Inf/NaN entries; the reference's eigvals throws there)");
  return HYQ_OK;
}

int hyq_get_SC(hyq_ctx* ctx, double* S, double* C) {
  if (!ctx) return fail(nullptr, HYQ_EINVAL, "null ctx");
  HQ_CHECK(ctx, cudaSetDevice(ctx->device));
  const size_t b = sizeof(double) * 35 * ctx->N;
  // Fx/Fy are scratch between steps: reuse them for S and C
  launch_std_central(ctx->M, ctx->N, ctx->Fx, ctx->Fy, ctx->stream);
  HQ_CHECK(ctx, cudaGetLastError());
  if (S) HQ_CHECK(ctx, cudaMemcpyAsync(S, ctx->Fx, b, cudaMemcpyDeviceToHost, ctx->stream));
  if (C) HQ_CHECK(ctx, cudaMemcpyAsync(C, ctx->Fy, b, cudaMemcpyDeviceToHost, ctx->stream));
  HQ_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  return HYQ_OK;
}

#define CELLS_LAUNCH_CHECK()                                    \
  do {                                                          \
    cudaError_t e_ = cudaGetLastError();                        \
    if (e_ != cudaSuccess) return cuda_fail(nullptr, e_, "launch"); \
  } while (0)

int hyq_cells_flux_closure(const double* M, int64_t n, int32_t flag2D, double Ma, double* Fx, double* Fy, double* Fz, double* Mr, void* stream) {
  if (!M || n <= 0) return fail(nullptr, HYQ_EINVAL, "bad argument");
  launch_cells_flux(M, n, flag2D, Ma, Fx, Fy, Fz, Mr, (cudaStream_t)stream);
  CELLS_LAUNCH_CHECK();
  return HYQ_OK;
}
int hyq_cells_eigenvalues(const double* M, int64_t n, int32_t axis, int32_t flag2D, double Ma, int32_t positivity, double* v, double* Mr,
                          void* stream) {
  if (!M || !v || !Mr || n <= 0 || axis < 1 || axis > 3) return fail(nullptr, HYQ_EINVAL, "bad argument");
  launch_cells_eig(M, n, axis, flag2D, Ma, positivity, v, Mr, (cudaStream_t)stream);
  CELLS_LAUNCH_CHECK();
  return HYQ_OK;
}
int hyq_cells_closure_eigs(const double* mom, int64_t n, double* v, void* stream) {
  if (!mom || !v || n <= 0) return fail(nullptr, HYQ_EINVAL, "bad argument");
  launch_cells_closure_eigs(mom, n, v, (cudaStream_t)stream);
  CELLS_LAUNCH_CHECK();
  return HYQ_OK;
}
int hyq_cells_collision(const double* M, int64_t n, double dt, double Kn, int32_t positivity, double* out, void* stream) {
  if (!M || !out || n <= 0) return fail(nullptr, HYQ_EINVAL, "bad argument");
  launch_cells_collision(M, n, dt, Kn, positivity, out, (cudaStream_t)stream);
  CELLS_LAUNCH_CHECK();
  return HYQ_OK;
}
int hyq_cells_wavespeed_targets(const double* M, int64_t n, int32_t flag2D, double Ma, int32_t positivity, float* T, double* Mr, void* stream) {
  if (!M || !T || n <= 0) return fail(nullptr, HYQ_EINVAL, "bad argument");
  launch_cells_targets(M, n, flag2D, Ma, positivity, T, Mr, (cudaStream_t)stream);
  CELLS_LAUNCH_CHECK();
  return HYQ_OK;
}
int hyq_cells_phase_A(const double* M, int64_t n, int32_t flag2D, double Ma, int32_t positivity, double* Fx, double* Fy, double* Fz, double* Mr,
                      double* vp, void* stream) {
  if (!M || !Fx || !Fy || !Fz || !Mr || !vp || n <= 0) return fail(nullptr, HYQ_EINVAL, "bad argument");
  launch_cells_phase_A(M, n, flag2D, Ma, positivity, Fx, Fy, Fz, Mr, vp, (cudaStream_t)stream);
  CELLS_LAUNCH_CHECK();
  return HYQ_OK;
}

// ------------------------------------------------------ batched domains
// Every member is an ordinary context (own buffers, stream, clock and step
// graph); the batch graph holds each member's step graph as an independent
// child node, so one replay advances all members by one step each and the
// kernels of small grids run side by side instead of one grid at a time.
// (Chaining several steps per member inside one graph measured slower on
// the 64-domain sweep: the large members' chains then run alone at the end
// of every replay.)
struct hyq_batch {
  std::vector<hyq_ctx*> sims;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t replayed = nullptr;  // recorded after each hyq_batch_advance_async
  int schedule = HYQ_BATCH_FUSED;
  int hll_variant = 0;
  int corr_variant = 0;
  // fused schedule: the member table and the block prefixes of each launch
  // kind on the device
  Dom* d_dom = nullptr;
  int* d_blk = nullptr;
  BatchPlan plan{};
  std::vector<int> gens;  // the members' graph generations at the last capture
};

namespace {
// correction passes: blocks per member of a fused launch, by variant
constexpr int CORR_CAPS[HYQ_CORR_VARIANTS] = {64, 16, 4, CORR_BLOCKS};

bool batch_fusable(const hyq_batch* b) {
  for (const hyq_ctx* c : b->sims)
    if (c->sc.mode != b->sims[0]->sc.mode) return false;
  return true;
}

// The member table and block prefixes of the fused launches, on the device.
int batch_plan(hyq_batch* b) {
  const int n = (int)b->sims.size();
  std::vector<Dom> dom(n);
  std::vector<int> blk((size_t)DK_NKIND * (n + 1), 0);
  for (int m = 0; m < n; ++m) {
    const hyq_ctx* c = b->sims[m];
    Dom& d = dom[m];
    d.sc = c->sc;
    d.clk = c->clk;
    d.buf[DB_M] = c->M; d.buf[DB_MTMP] = c->Mtmp; d.buf[DB_FX] = c->Fx; d.buf[DB_FY] = c->Fy; d.buf[DB_FZ] = c->Fz;
    d.buf[DB_VP] = c->vp; d.buf[DB_BMAX] = c->blockmax;
    int nb[DK_NKIND];
    dom_blocks(c->sc.Nx, c->sc.Ny, c->sc.Nz, b->hll_variant, CORR_CAPS[b->corr_variant], nb);
    for (int k = 0; k < DK_NKIND; ++k) {
      const long long next = (long long)blk[(size_t)k * (n + 1) + m] + nb[k];
      if (next > 0x7fffffffLL) return fail(nullptr, HYQ_EINVAL, "fused batch: too many blocks in one launch");
      blk[(size_t)k * (n + 1) + m + 1] = (int)next;
    }
  }
  cudaError_t e;
  if (!b->d_dom) {
    if ((e = cudaMalloc((void**)&b->d_dom, sizeof(Dom) * n)) != cudaSuccess) return cuda_fail(nullptr, e, "batch member table");
    if ((e = cudaMalloc((void**)&b->d_blk, sizeof(int) * blk.size())) != cudaSuccess) return cuda_fail(nullptr, e, "batch block table");
  }
  if ((e = cudaMemcpyAsync(b->d_dom, dom.data(), sizeof(Dom) * n, cudaMemcpyHostToDevice, b->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(b->d_blk, blk.data(), sizeof(int) * blk.size(), cudaMemcpyHostToDevice, b->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(b->stream)) != cudaSuccess)
    return cuda_fail(nullptr, e, "batch tables");
  b->plan.dom = b->d_dom;
  b->plan.n = n;
  b->plan.hll_variant = b->hll_variant;
  for (int k = 0; k < DK_NKIND; ++k) {
    b->plan.blk0[k] = b->d_blk + (size_t)k * (n + 1);
    b->plan.nblk[k] = blk[(size_t)k * (n + 1) + n];
  }
  return HYQ_OK;
}

// The learned path's network launches of every member, after the fused
// first closure (each member's own weights and seed buffer).
void batch_seeds(void* arg, cudaStream_t s) {
  const hyq_batch* b = static_cast<const hyq_batch*>(arg);
  for (const hyq_ctx* c : b->sims) launch_wavespeed_seeds(c->sc, c->Fx, &c->net, c->sc.seeds, c->clk, s, 0, c->N);
}

// One graph per step: the fused launches, or the members' step graphs as
// independent branches.
int batch_capture(hyq_batch* b) {
  cudaError_t e;
  for (const hyq_ctx* c : b->sims)
    if (c->sc.mode == MODE_LEARNED && !c->net_loaded)
      return fail(nullptr, HYQ_EINVAL, "HYQ_MODE_LEARNED members need their wave-speed networks (hyq_set_wavespeed_net) first");
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  if (b->schedule == HYQ_BATCH_FUSED) {
    const int r = batch_plan(b);
    if (r != HYQ_OK) return r;
    const int mode = b->sims[0]->sc.mode;
    if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return cuda_fail(nullptr, e, "cudaStreamBeginCapture");
    launch_phase_A_batch(b->plan, mode, b->stream, mode == MODE_LEARNED ? batch_seeds : nullptr, b);
    launch_mid_batch(b->plan, b->stream);
    launch_phase_EF_batch(b->plan, mode, b->stream);
    launch_maxdiff_batch(b->plan, b->stream);
    if ((e = cudaStreamEndCapture(b->stream, &b->graph)) != cudaSuccess) return cuda_fail(nullptr, e, "cudaStreamEndCapture");
  } else {
    if ((e = cudaGraphCreate(&b->graph, 0)) != cudaSuccess) return cuda_fail(nullptr, e, "batch graph");
    // largest members first, so that their kernels start first and the small
    // members' kernels fill the SMs they leave free
    std::vector<hyq_ctx*> order(b->sims);
    std::stable_sort(order.begin(), order.end(), [](const hyq_ctx* x, const hyq_ctx* y) { return x->N > y->N; });
    for (hyq_ctx* c : order) {
      cudaGraphNode_t node;
      if ((e = cudaGraphAddChildGraphNode(&node, b->graph, nullptr, 0, c->graph)) != cudaSuccess)
        return cuda_fail(nullptr, e, "cudaGraphAddChildGraphNode");
    }
  }
  if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) return cuda_fail(nullptr, e, "cudaGraphInstantiate");
  b->gens.clear();
  for (const hyq_ctx* c : b->sims) b->gens.push_back(c->gen);
  return HYQ_OK;
}

// Capture again when a member's constants or graph changed since.
int batch_refresh(hyq_batch* b) {
  bool stale = !b->exec || b->gens.size() != b->sims.size();
  for (size_t m = 0; !stale && m < b->sims.size(); ++m) stale = b->gens[m] != b->sims[m]->gen;
  return stale ? batch_capture(b) : HYQ_OK;
}
}  // namespace

void hyq_batch_destroy(hyq_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->replayed) cudaEventDestroy(b->replayed);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_dom) cudaFree(b->d_dom);
  if (b->d_blk) cudaFree(b->d_blk);
  if (b->stream) cudaStreamDestroy(b->stream);
  for (hyq_ctx* c : b->sims) hyq_destroy(c);
  delete b;
}

int hyq_batch_create(const hyq_params* p, int32_t n, hyq_batch** out) {
  if (!p || !out || n < 1) return fail(nullptr, HYQ_EINVAL, "null argument or empty batch");
  if (n > DK_MAX_MEMBERS) return fail(nullptr, HYQ_EINVAL, "too many members for one batch");
  *out = nullptr;
  for (int32_t i = 1; i < n; ++i)
    if (p[i].device != p[0].device) return fail(nullptr, HYQ_EINVAL, "all members of a batch must use the same device");
  hyq_batch* b = new hyq_batch();
  b->device = p[0].device;
  for (int32_t i = 0; i < n; ++i) {
    hyq_ctx* c = nullptr;
    const int r = hyq_create(&p[i], &c);
    if (r != HYQ_OK) {
      const std::string msg = "member " + std::to_string(i) + ": " + g_err;
      hyq_batch_destroy(b);
      return fail(nullptr, r, msg);
    }
    b->sims.push_back(c);
  }
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&b->replayed, cudaEventDisableTiming)) != cudaSuccess) {
    const int r = cuda_fail(nullptr, e, "batch stream");
    hyq_batch_destroy(b);
    return r;
  }
  if (!batch_fusable(b)) b->schedule = HYQ_BATCH_BRANCHES;
  // learned members are captured at the first advance, after their networks
  if (b->sims[0]->sc.mode != MODE_LEARNED) {
    const int r = batch_capture(b);
    if (r != HYQ_OK) {
      hyq_batch_destroy(b);
      return r;
    }
  }
  *out = b;
  return HYQ_OK;
}

int hyq_batch_set_schedule(hyq_batch* b, int32_t schedule) {
  if (!b) return fail(nullptr, HYQ_EINVAL, "null batch");
  if (schedule != HYQ_BATCH_FUSED && schedule != HYQ_BATCH_BRANCHES) return fail(nullptr, HYQ_EINVAL, "unknown schedule");
  if (schedule == HYQ_BATCH_FUSED && !batch_fusable(b))
    return fail(nullptr, HYQ_EINVAL, "a fused batch needs one eigenvalue path (hyq_params.mode) for all members");
  HQ_CHECK(nullptr, cudaSetDevice(b->device));
  HQ_CHECK(nullptr, cudaStreamSynchronize(b->stream));
  b->schedule = schedule;
  return batch_capture(b);
}

int32_t hyq_batch_schedule(const hyq_batch* b) { return b ? b->schedule : -1; }

int hyq_batch_set_variant(hyq_batch* b, int32_t kernel, int32_t variant) {
  if (!b) return fail(nullptr, HYQ_EINVAL, "null batch");
  if (variant < 0 || variant >= hyq_variant_count(kernel)) return fail(nullptr, HYQ_EINVAL, "unknown kernel or variant out of range");
  HQ_CHECK(nullptr, cudaSetDevice(b->device));
  HQ_CHECK(nullptr, cudaStreamSynchronize(b->stream));
  if (kernel == HYQ_KERNEL_HLL) {
    b->hll_variant = variant;
    for (hyq_ctx* c : b->sims) {
      const int r = hyq_set_variant(c, kernel, variant);
      if (r != HYQ_OK) return fail(nullptr, r, c->err);
    }
  } else {
    b->corr_variant = variant;
  }
  return batch_capture(b);
}

int32_t hyq_batch_size(const hyq_batch* b) { return b ? (int32_t)b->sims.size() : 0; }

hyq_ctx* hyq_batch_member(hyq_batch* b, int32_t i) {
  if (!b || i < 0 || i >= (int32_t)b->sims.size()) return nullptr;
  return b->sims[i];
}

void* hyq_batch_stream(hyq_batch* b) { return b ? (void*)b->stream : nullptr; }

int hyq_batch_advance_async(hyq_batch* b, int64_t max_steps) {
  if (!b || max_steps < 0) return fail(nullptr, HYQ_EINVAL, "bad argument");
  HQ_CHECK(nullptr, cudaSetDevice(b->device));
  // members' own streams may still hold a state upload or clock reset
  for (hyq_ctx* c : b->sims) HQ_CHECK(nullptr, cudaStreamSynchronize(c->stream));
  for (hyq_ctx* c : b->sims)
    if (c->sc.mode == MODE_LEARNED && !c->net_loaded)
      return fail(nullptr, HYQ_EINVAL, "HYQ_MODE_LEARNED members need their wave-speed networks before stepping");
  const int r = batch_refresh(b);
  if (r != HYQ_OK) return r;
  for (int64_t s = 0; s < max_steps; ++s) HQ_CHECK(nullptr, cudaGraphLaunch(b->exec, b->stream));
  // member calls run on the members' own streams: order them after the replays
  HQ_CHECK(nullptr, cudaEventRecord(b->replayed, b->stream));
  for (hyq_ctx* c : b->sims) HQ_CHECK(nullptr, cudaStreamWaitEvent(c->stream, b->replayed, 0));
  return HYQ_OK;
}

int hyq_batch_advance(hyq_batch* b, int64_t max_steps, int32_t* ndone, int32_t* nfailed) {
  int r = hyq_batch_advance_async(b, max_steps);
  if (r) return r;
  HQ_CHECK(nullptr, cudaStreamSynchronize(b->stream));
  int32_t done = 0, failed = 0;
  for (hyq_ctx* c : b->sims) {
    hyq_stats st;
    if ((r = hyq_stats_get(c, &st)) != HYQ_OK) return fail(nullptr, r, c->err);
    done += st.done ? 1 : 0;
    failed += st.status > 0 ? 1 : 0;
  }
  if (ndone) *ndone = done;
  if (nfailed) *nfailed = failed;
  return HYQ_OK;
}

}  // extern "C"
