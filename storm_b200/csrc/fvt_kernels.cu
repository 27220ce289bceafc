// fvt_kernels.cu -- sm_100a kernels of one SToRM FVT iteration (solverFVT.f90:129-476).
//
// One RK stage (solverFVT.f90:161-325) is:
//   k_node   per node : ctr2vtxWSE type 3 + cap + positivity_vtx + enforce_bcs stage
//                       nodes (to_vertices.f90:26-41, enforce_bcs.f90:37-56)
//   k_grad   per cell : find_dry_cells state, lsq_grad_array x3, limiterBJ x3, delh -= delz
//                       (cell_grads.f90), hgradfix2.f90:48-98, zeroing of cells with a
//                       vertex depth <= h_dry (to_vertices.f90:44-55)
//   k_bc     per open boundary (one CTA): inflowQbyH / inflowH / outflowbyH /
//                       crit_outflow / free_flow, including the inflow fixed point
//   k_eflux  per interior edge: the Roe/HLL/Rusanov flux (with the I1 wet/dry wall test)
//                       evaluated once, in the reference's orientation, times the length
//   k_flux   per cell : the cell's face contributions (edge fluxes from k_eflux, the
//                       wenslp3/weslp2 walls, boundary contributions) added in the order
//                       invisc_fluxes.f90 scatters them, bed_slope_STD + adjustZb, the
//                       SSP-RK combination, vclip, h >= 0 and wet/dry hysteresis
//                       (k_flux_bc: the cells with an open-boundary face, after k_bc)
// and one iteration ends with
//   k_fric  per cell : find_dry_cells, fric_terms_impl, the numerical valve, the
//                      RK level copy, block partials of sumtop/sumbot/tmass/max|phi|/dt
//   k_final one CTA per scenario: deterministic reduction of the partials, stop test,
//                      clocks, get_time_bcs.
// No float atomics: every sum is a fixed-order tree or a serial loop, so the results
// are reproducible run to run.
#include <cstdint>
#include <mutex>

#include "fvt_device.cuh"
#include "storm_internal.h"

namespace storm {

namespace {

constexpr double kZero = 0.0;
constexpr double kHalf = 0.5;
constexpr double kOne = 1.0;
constexpr double kOneThird = 1.0 / 3.0;
constexpr double kG = 9.81;
constexpr double kFmachp = 2.220446049250313e-16;   // EPSILON(zero)
constexpr double kVsmall = 2.2250738585072014e-308; // TINY(zero)
constexpr double kVlarge = 1.7976931348623157e+308; // HUGE(zero)
#define SMALL_F ((double)1.0e-9f)                   // REAL(mp) :: small = 1.0E-9

__device__ __forceinline__ double fmin2(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double fmax2(double a, double b) { return (b > a) ? b : a; }

// The IEEE quotient a / b, with a zero numerator answered without the division: for
// a nonzero b that is not a NaN, a signed zero divided by b is the zero whose sign is
// the exclusive or of the two signs, which is exactly what the division returns.  A
// zero quotient is rare in general code but common here (dry cells, still water, a
// limiter ratio whose numerator is the cell's own extremum, axis-aligned normals),
// and the division's own handling of that case costs far more than this test.
__device__ __forceinline__ double qdiv(double a, double b) {
  double r;
  if (a == 0.0 && b != 0.0 && b == b)
    r = __longlong_as_double((__double_as_longlong(a) ^ __double_as_longlong(b)) &
                             (long long)0x8000000000000000ULL);
  else
    r = a / b;
  return r;
}
// The mixed path's FP32 quotients: the approximate reciprocal-multiply division
// (__fdividef, within 2 ulp for |b| in [2^-126, 2^126]; the denominators here are
// determinants, celerities, wave-speed spans and limiter increments of ordinary
// magnitude), whose error is far below the FP32 rounding the path already accepts.
__device__ __forceinline__ float qdiv(float a, float b) { return __fdividef(a, b); }

// sqrt with a zero argument answered directly (sqrt(+-0) = +-0 under IEEE), for the
// same reason as qdiv: still water and dry sides make zero arguments common.
__device__ __forceinline__ double qsqrt(double x) {
  double r = x;
  if (x != 0.0) r = sqrt(x);
  return r;
}
__device__ __forceinline__ float qsqrt(float x) {
  float r = x;
  if (x != 0.0f) r = sqrtf(x);
  return r;
}

// equals.f90:1-27
__device__ __forceinline__ bool equals(double a, double b) {
  double eps = fabs(a) * kFmachp;
  if (eps == kZero) eps = kVsmall;
  return !(fabs(a - b) > eps);
}

// find_dry_cells.f90:25-42 for one cell; returns drycell and writes u_mag.
__device__ __forceinline__ bool dry_flag(double h, double u, double v, double h_dry, double h_wet,
                                         double* umag) {
  bool dry = h < h_dry;
  double um = kZero;
  if (!dry) um = qsqrt(u * u + v * v);
  *umag = um;
  if (!dry && (h < h_wet) && equals(um, kZero)) dry = true;
  return dry;
}

// Whether cell slot c (node n, edge e) belongs to a scenario that is still running.
// A one-scenario handle answers from the slot number and one flag shared by every
// thread, so a thread's own loads do not wait behind a per-cell scenario lookup; a
// batch looks up the slot's scenario (-1: padding).
__device__ __forceinline__ bool cell_live(const Dev& d, int c) {
  if (d.nscen == 1) return c < d.t_real && !d.sc[0].converged;
  const int sid = d.cell_sid[c];
  return sid >= 0 && !d.sc[sid].converged;
}
// Scenario of a live cell (one-scenario handles: 0, without the lookup).
__device__ __forceinline__ int cell_scenario(const Dev& d, int c) { return d.nscen == 1 ? 0 : d.cell_sid[c]; }
__device__ __forceinline__ bool item_live(const Dev& d, const int32_t* __restrict__ sid_of, int i) {
  if (d.nscen == 1) return !d.sc[0].converged;
  return !d.sc[sid_of[i]].converged;
}

// Arithmetic type of the flux, gradient and source kernels: double reproduces the
// reference bit for bit; float is the mixed-precision path (state, the eta - zb
// reconstruction at the faces and the RK accumulation stay in double).
__device__ __forceinline__ float fmin2(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fmax2(float a, float b) { return (b > a) ? b : a; }
// x + 0: the first step of each MATMUL sum (turns a -0 product into +0)
__device__ __forceinline__ double add0(double x) { return __dadd_rn(x, 0.0); }
__device__ __forceinline__ float add0(float x) { return __fadd_rn(x, 0.0f); }

// flux_ac.f90:48-126.  The MATMULs start from zero and add x(i,k)*y(k,j) for
// k = 1..3; with the diagonal eigenvalue matrix (entries >= delta > 0) the first
// product reduces exactly to rev(i,j)*eigv(j) + 0.
template <class R>
__device__ __forceinline__ void flux_roe(R nx, R ny, R hleft, R uleft, R vleft, R hright, R uright, R vright,
                                         R* flux) {
  const R delta = R(0.10);
  R fl[3], gl[3], fr[3], gr[3];
  fl[0] = hleft * uleft;
  fl[1] = hleft * uleft * uleft + R(kHalf) * R(kG) * hleft * hleft;
  fl[2] = hleft * uleft * vleft;
  gl[0] = hleft * vleft;
  gl[1] = hleft * uleft * vleft;
  gl[2] = hleft * vleft * vleft + R(kHalf) * R(kG) * hleft * hleft;
  fr[0] = hright * uright;
  fr[1] = hright * uright * uright + R(kHalf) * R(kG) * hright * hright;
  fr[2] = hright * uright * vright;
  gr[0] = hright * vright;
  gr[1] = hright * uright * vright;
  gr[2] = hright * vright * vright + R(kHalf) * R(kG) * hright * hright;
  hleft = fmax2(hleft, R(SMALL_F));
  R hls = sqrt(hleft);
  hright = fmax2(hright, R(SMALL_F));
  R hrs = sqrt(hright);
  R denom = hrs + hls;
  R uavg = qdiv(uright * hrs + uleft * hls, denom);
  R vavg = qdiv(vright * hrs + vleft * hls, denom);
  R cavg = sqrt(R(kHalf) * R(kG) * (hleft + hright));
  R q[3];
  q[0] = hright - hleft;
  q[1] = hright * uright - hleft * uleft;
  q[2] = hright * vright - hleft * vleft;
  R rev[3][3], lev[3][3], t1[3][3], eig[3];
  rev[0][0] = R(kZero); rev[0][1] = R(kOne); rev[0][2] = R(kOne);
  rev[1][0] = ny; rev[1][1] = uavg - cavg * nx; rev[1][2] = uavg + cavg * nx;
  rev[2][0] = -nx; rev[2][1] = vavg - cavg * ny; rev[2][2] = vavg + cavg * ny;
  lev[0][0] = -(uavg * ny - vavg * nx);
  lev[0][1] = ny;
  lev[0][2] = -nx;
  lev[1][0] = qdiv(R(kHalf) * (uavg * nx + vavg * ny), cavg) + R(kHalf);
  lev[1][1] = -qdiv(R(kHalf) * nx, cavg);
  lev[1][2] = -qdiv(R(kHalf) * ny, cavg);
  lev[2][0] = -qdiv(R(kHalf) * (uavg * nx + vavg * ny), cavg) + R(kHalf);
  lev[2][1] = qdiv(R(kHalf) * nx, cavg);
  lev[2][2] = qdiv(R(kHalf) * ny, cavg);
  eig[0] = fmax2(fabs(uavg * nx + vavg * ny), delta);
  eig[1] = fmax2(fabs(uavg * nx + vavg * ny - cavg), delta);
  eig[2] = fmax2(fabs(uavg * nx + vavg * ny + cavg), delta);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) t1[i][j] = add0(rev[i][j] * eig[j]);
  R aq[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    R t2[3];
#pragma unroll
    for (int j = 0; j < 3; j++)
      t2[j] = (add0(t1[i][0] * lev[0][j]) + t1[i][1] * lev[1][j]) + t1[i][2] * lev[2][j];
    aq[i] = (add0(t2[0] * q[0]) + t2[1] * q[1]) + t2[2] * q[2];
  }
#pragma unroll
  for (int i = 0; i < 3; i++) flux[i] = R(kHalf) * (fr[i] * nx + gr[i] * ny + fl[i] * nx + gl[i] * ny - aq[i]);
}

// flux_HLL.f90:41-110 with its two defects fixed (flux(3) assigned; the whole HLL
// numerator divided by sright - sleft).  The debug stop at :88-91 sets *bad.
template <class R>
__device__ __forceinline__ void flux_hll(R nx, R ny, R hleft, R uleft, R vleft, R hright, R uright, R vright,
                                         R h0, R* flux, bool* bad) {
  R cleft = qsqrt(R(kG) * hleft);
  R cright = qsqrt(R(kG) * hright);
  R ustar = R(kHalf) * ((uleft + uright) * nx + (vleft + vright) * ny) + cleft - cright;
  R cstar = R(kHalf) * (cleft + cright) + ((uleft - uright) * nx + (vleft - vright) * ny) / R(4.0);
  R sleft, sright, aux1, aux2;
  if (hleft < h0) sleft = uright * nx + vright * ny - R(2.0) * cright;
  else if (hright < h0) sleft = uleft * nx + vleft * ny - cleft;
  else {
    aux1 = uleft * nx + vleft * ny - cleft;
    aux2 = ustar - cstar;
    sleft = fmin2(aux1, aux2);
  }
  if (hleft < h0) sright = uright * nx + vright * ny + cright;
  else if (hright < h0) sright = uleft * nx + vleft * ny + R(2.0) * cleft;
  else {
    aux1 = uright * nx + vright * ny - cright;
    aux2 = ustar + cstar;
    sright = fmax2(aux1, aux2);
  }
  R fl[3], gl[3], fr[3], gr[3];
  fl[0] = hleft * uleft * nx;
  fl[1] = (hleft * uleft * uleft + R(kHalf) * R(kG) * hleft * hleft) * nx;
  fl[2] = hleft * uleft * vleft * nx;
  gl[0] = hleft * vleft * ny;
  gl[1] = hleft * uleft * vleft * ny;
  gl[2] = (hleft * vleft * vleft + R(kHalf) * R(kG) * hleft * hleft) * ny;
  fr[0] = hright * uright * nx;
  fr[1] = (hright * uright * uright + R(kHalf) * R(kG) * hright * hright) * nx;
  fr[2] = hright * uright * vright * nx;
  gr[0] = hright * vright * ny;
  gr[1] = hright * uright * vright * ny;
  gr[2] = (hright * vright * vright + R(kHalf) * R(kG) * hright * hright) * ny;
  if (sleft > R(kZero) && sright < R(kZero)) *bad = true;
  if (sleft > R(kZero)) {
    for (int i = 0; i < 3; i++) flux[i] = fl[i] + gl[i];
  } else if (sright < R(kZero)) {
    for (int i = 0; i < 3; i++) flux[i] = fr[i] + gr[i];
  } else {
    aux1 = sright - sleft;
    flux[0] = qdiv(sright * (fl[0] + gl[0]) - sleft * (fr[0] + gr[0]) + sleft * sright * (hright - hleft), aux1);
    flux[1] = qdiv(sright * (fl[1] + gl[1]) - sleft * (fr[1] + gr[1]) +
                       sleft * sright * (hright * uright - hleft * uleft), aux1);
    flux[2] = qdiv(sright * (fl[2] + gl[2]) - sleft * (fr[2] + gr[2]) +
                       sleft * sright * (hright * vright - hleft * vleft), aux1);
  }
}

// flux_rusanov.f90:47-80
template <class R>
__device__ __forceinline__ void flux_rusanov(R nx, R ny, R hleft, R uleft, R vleft, R cl, R hright, R uright,
                                             R vright, R cr, R* flux) {
  R fl[3], gl[3], fr[3], gr[3], q[3];
  fl[0] = hleft * uleft;
  fl[1] = hleft * uleft * uleft + R(kHalf) * R(kG) * hleft * hleft;
  fl[2] = hleft * uleft * vleft;
  gl[0] = hleft * vleft;
  gl[1] = hleft * uleft * vleft;
  gl[2] = hleft * vleft * vleft + R(kHalf) * R(kG) * hleft * hleft;
  fr[0] = hright * uright;
  fr[1] = hright * uright * uright + R(kHalf) * R(kG) * hright * hright;
  fr[2] = hright * uright * vright;
  gr[0] = hright * vright;
  gr[1] = hright * uright * vright;
  gr[2] = hright * vright * vright + R(kHalf) * R(kG) * hright * hright;
  R ul = uleft * nx + vleft * ny;
  R ur = uright * nx + vright * ny;
  R splus = fmax2(fabs(ul) + cl, fabs(ur) + cr);
  q[0] = hright - hleft;
  q[1] = hright * uright - hleft * uleft;
  q[2] = hright * vright - hleft * vleft;
#pragma unroll
  for (int i = 0; i < 3; i++) flux[i] = R(kHalf) * (fr[i] * nx + gr[i] * ny + fl[i] * nx + gl[i] * ny - splus * q[i]);
}

// Block-level reductions in a fixed order (warp xor-shuffle tree, then warps in order).
template <int NT>
__device__ __forceinline__ double block_sum(double x, double* sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = x + __shfl_xor_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sm[w] = x;
  __syncthreads();
  double r = kZero;
  if (threadIdx.x == 0) {
    r = sm[0];
    for (int i = 1; i < NT / 32; i++) r = r + sm[i];
  }
  return r;  // valid on thread 0
}
template <int NT>
__device__ __forceinline__ double block_max(double x, double* sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmax2(x, __shfl_xor_sync(0xffffffffu, x, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sm[w] = x;
  __syncthreads();
  double r = kZero;
  if (threadIdx.x == 0) {
    r = sm[0];
    for (int i = 1; i < NT / 32; i++) r = fmax2(r, sm[i]);
  }
  return r;
}
template <int NT>
__device__ __forceinline__ double block_min(double x, double* sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmin2(x, __shfl_xor_sync(0xffffffffu, x, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sm[w] = x;
  __syncthreads();
  double r = kZero;
  if (threadIdx.x == 0) {
    r = sm[0];
    for (int i = 1; i < NT / 32; i++) r = fmin2(r, sm[i]);
  }
  return r;
}

// The five iteration reductions in one pass: sums of st, sb, tm, the max of rm and the
// min of dt, each by the same xor-shuffle tree and the same serial warp order as
// block_sum / block_max / block_min (so the same bits), with one barrier.
template <int NT>
__device__ __forceinline__ void block_reduce5(double st, double sb, double tm, double rm, double dt, double* sm,
                                              double* out, size_t os = 1) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    st = st + __shfl_xor_sync(0xffffffffu, st, o);
    sb = sb + __shfl_xor_sync(0xffffffffu, sb, o);
    tm = tm + __shfl_xor_sync(0xffffffffu, tm, o);
    rm = fmax2(rm, __shfl_xor_sync(0xffffffffu, rm, o));
    dt = fmin2(dt, __shfl_xor_sync(0xffffffffu, dt, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  constexpr int NW = NT / 32;
  __syncthreads();
  if (l == 0) {
    sm[w] = st;
    sm[NW + w] = sb;
    sm[2 * NW + w] = tm;
    sm[3 * NW + w] = rm;
    sm[4 * NW + w] = dt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = sm[0], b = sm[NW], c = sm[2 * NW], m = sm[3 * NW], n = sm[4 * NW];
    for (int i = 1; i < NW; i++) {
      a = a + sm[i];
      b = b + sm[NW + i];
      c = c + sm[2 * NW + i];
      m = fmax2(m, sm[3 * NW + i]);
      n = fmin2(n, sm[4 * NW + i]);
    }
    out[0] = a;
    out[os] = b;
    out[2 * os] = c;
    out[3 * os] = m;
    out[4 * os] = n;
  }
}

// get_time_bcs.f90:31-77 for scenario `sid` (one thread)
__device__ void time_bcs(const Dev& d, int sid, double time) {
  Scalars* sc = &d.sc[sid];
  for (int k = 0; k < sc->n_out; k++) {
    if (sc->out_type[k] != 1) continue;
    int n = sc->ts_cnt[kMaxBdrDev + k];
    if (n <= 0) continue;
    const double* tl = d.ts_t + sc->ts_off[kMaxBdrDev + k];
    const double* ts = d.ts_v + sc->ts_off[kMaxBdrDev + k];
    if (time < tl[0]) sc->hbc[k] = ts[0];
    else if (time >= tl[n - 1]) sc->hbc[k] = ts[n - 1];
    else
      for (int i = 0; i < n - 1; i++)
        if (time >= tl[i] && time < tl[i + 1]) {
          double delta = time - tl[i], delta2 = tl[i + 1] - tl[i];
          sc->hbc[k] = ts[i] + delta * (ts[i + 1] - ts[i]) / delta2;
          break;
        }
  }
  for (int k = 0; k < sc->n_in; k++) {
    int n = sc->ts_cnt[k];
    if (n <= 0) continue;
    const double* tl = d.ts_t + sc->ts_off[k];
    const double* ts = d.ts_v + sc->ts_off[k];
    if (time < tl[0]) sc->qin[k] = ts[0];
    else if (time >= tl[n - 1]) sc->qin[k] = ts[n - 1];
    else
      for (int j = 0; j < n - 1; j++)
        if (time >= tl[j] && time < tl[j + 1]) {
          double delta = time - tl[j], delta2 = tl[j + 1] - tl[j];
          sc->qin[k] = ts[j] + delta * (ts[j + 1] - ts[j]) / delta2;
          break;
        }
  }
}

}  // namespace

// The FP32 (mixed-precision) instantiations of the stage and output kernels live in
// fvt_kernels_f32.cu, a second compilation of this file with FMA contraction allowed:
// the FP64 path keeps every operation rounded as written, the mixed path needs no
// such order.  These are its entry points.
int tile_blocks_per_sm_f32(size_t smem);
void set_tile_smem_attr_f32(int bytes);
void set_bc_smem_attr_f32(int bytes);
void launch_stage_f32(const StageLaunch& L, const Dev& d, const Geo<float>& G);
void launch_out_cell_f32(const Dev& d, const Geo<float>& G, const OutputArgs& a, int grid, cudaStream_t st);

constexpr int kRedThreads = 256;
constexpr int kFinalThreads = 512;  // k_final: one CTA per scenario over its block partials

#ifndef STORM_FVT_F32_TU
// ---------------------------------------------------------------------------
// Initial state: rk(:,0) = (h, h*u, h*v) (solverFVT.f90:122-126 then :138-142),
// first-stage dry flags and the CFL dt partials of the initial state.
__global__ void __launch_bounds__(kRedThreads) k_init(Dev d, int c0) {
  __shared__ double sm[kRedThreads / 32];
  const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  double dtc = kVlarge;
  if (c < d.T && d.cell_sid[c] >= 0) {
    double h = d.rkh[c], u = d.u_a[c], v = d.v_a[c];
    d.rku[c] = h * u;
    d.rkv[c] = h * v;
    double um;
    bool dry = dry_flag(h, u, v, d.h_dry, d.h_wet, &um);
    d.dry_a[c] = dry;
    double wc = dry ? kZero : sqrt(kG * h);
    double dl = um + wc + SMALL_F;
    dtc = d.cfl * d.area[c] / (dl * d.perim[c]);
  }
  double r = block_min<kRedThreads>(dtc, sm);
  if (threadIdx.x == 0) d.part[4 * (size_t)d.nblk_red + c0 / kRedThreads + blockIdx.x] = r;
}

// One block per listed scenario: initial scalars and the first dt.
__global__ void __launch_bounds__(kRedThreads) k_init_final(Dev d, int sid) {
  __shared__ double sm[kRedThreads / 32];
  Scalars* sc = &d.sc[sid];
  double m = kVlarge;
  for (int b = threadIdx.x; b < sc->blk_cnt; b += blockDim.x) m = fmin2(m, d.part[4 * (size_t)d.nblk_red + sc->blk_off + b]);
  double dtmin = block_min<kRedThreads>(m, sm);
  if (threadIdx.x == 0) {
    sc->iter = 0;
    sc->converged = 0;
    sc->status = 0;
    sc->ttime = kZero;
    sc->stime = kZero;
    sc->rmax = kZero;
    sc->rms = kZero;
    sc->tmass = kZero;
    sc->delt_fric = kZero;
    for (int b = 0; b < kMaxBdrDev; b++) {
      sc->cqin3[b] = kZero;
      sc->cqout3[b] = kZero;
    }
    time_bcs(d, sid, kZero);
    for (int b = 0; b < kMaxBdrDev; b++) {
      sc->qin_it[b] = sc->qin[b];
      sc->hbc_it[b] = sc->hbc[b];
    }
    if (d.steady) sc->delt = kZero;  // delt is first set inside the RK loop
    else sc->delt = (d.dt_op == 0) ? d.cfl : dtmin;
  }
}
#endif  // !STORM_FVT_F32_TU

// ---------------------------------------------------------------------------
// Vertex water surface and depth of one stage (to_vertices.f90:26-41: ctr2vtxWSE type
// 3, cap at the highest wet neighbour, positivity_vtx; enforce_bcs.f90:37-56 for the
// stage nodes).  cell(q, &dry, &h, &z) gives the q-th incident cell (n2t order).
template <class CellF>
__device__ __forceinline__ void node_depth(const Dev& d, int n, int b0, int b1, CellF cell, double* hv_out,
                                           bool* wet_out) {
  const double zv0 = d.zvtx[n];
  double id = kZero, a = kZero, zetaref = zv0;
  int counter = 0;
  for (int q = b0; q < b1; q++) {
    bool dk;
    double hk, zk;
    cell(q, &dk, &hk, &zk);
    if (dk) continue;
    const double zeta = hk + zk;
    const double w = d.n2t_w[q];
    counter++;
    id = id + w;
    a = a + w * zeta;
    zetaref = fmax2(zeta, zetaref);
  }
  double zv = counter > 0 ? a / id : zv0;
  zv = fmin2(zv, zetaref);
  double hv = zv - zv0;
  if (hv < kZero) hv = kZero;
  *wet_out = hv > d.h_dry;
  const int b = d.node_hbc[n];
  if (b >= 0) hv = fmax2(kZero, d.sc[d.node_sid[n]].hbc[b] - zv0);
  *hv_out = hv;
}

#ifndef STORM_FVT_F32_TU
// Every node, or the listed nodes (the vertices of the cells with an open-boundary
// face, ahead of their gradients on the side stream of the fused path).
__global__ void __launch_bounds__(256) k_node(Dev d, const double* __restrict__ hs, const uint8_t* __restrict__ dry,
                                              const int32_t* __restrict__ list, int nlist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int n;
  if (list) {
    if (i >= nlist) return;
    n = list[i];
  } else {
    if (i >= d.N) return;
    n = i;
  }
  if (!item_live(d, d.node_sid, n)) return;
  double hv;
  bool wet;
  node_depth(d, n, d.n2t_off[n], d.n2t_off[n + 1],
             [&](int q, bool* dk, double* hk, double* zk) {
               const int k = d.n2t_cell[q];
               *dk = dry[k] != 0;
               *hk = hs[k];
               *zk = d.z[k];
             },
             &hv, &wet);
  d.vwet[n] = wet;
  d.hvtx[n] = hv;
}
#endif  // !STORM_FVT_F32_TU

// The face value of a cell field, x + grad . rc (invisc_fluxes.f90:58-64): in double as
// the reference writes it; on the mixed path the FP32 correction is added to the FP64
// value, so the depth at a wet/dry front keeps its eta - zb precision.
__device__ __forceinline__ double recon(double x, double gx, double rx, double gy, double ry) {
  return x + gx * rx + gy * ry;
}
__device__ __forceinline__ double recon(double x, float gx, float rx, float gy, float ry) {
  return x + (double)(gx * rx + gy * ry);
}

// ---------------------------------------------------------------------------
// Limited LSQ gradients, hgradfix2 and the partially-wet velocity zeroing
// (lsq_grad_array.f90:60-73, limiterBJ.f90:42-81 with beta = one, cell_grads.f90:72-75,
// hgradfix2.f90:48-98, to_vertices.f90:44-55).  Differences of the FP64 fields are
// taken in double and then rounded to R.
__device__ __forceinline__ double limited_r(double q0, double qn, double g_x, double g_y, double rx, double ry) {
  const double qmin = fmin2(q0, qn);
  const double qmax = fmax2(q0, qn);
  const double qj = q0 + g_x * rx + g_y * ry;
  const double delq = qj - q0;
  double rj;
  if (equals(delq, kZero)) rj = kOne;
  else {
    // r = (qmin-q0)/delq for delq < 0, (qmax-q0)/delq otherwise; both are >= 0.
    // When |num| > |delq| the exact quotient exceeds one, so the rounded one is
    // >= 1 and the limiter's min(r,1) is 1: the division is skipped, same bits.
    const double num = (delq < 0) ? (qmin - q0) : (qmax - q0);
    rj = (fabs(num) > fabs(delq)) ? kOne : qdiv(num, delq);
  }
  const double a = fmin2(kOne * rj, kOne);
  const double b = fmin2(rj, kOne);
  return fmax2(a, b);
}
__device__ __forceinline__ float limited_r(double q0, double qn, float g_x, float g_y, float rx, float ry) {
  const float dmin = (float)(fmin2(q0, qn) - q0), dmax = (float)(fmax2(q0, qn) - q0);
  const float delq = g_x * rx + g_y * ry;
  if (fabsf(delq) <= 1e-30f) return 1.0f;
  const float num = (delq < 0) ? dmin : dmax;
  return (fabsf(num) >= fabsf(delq)) ? 1.0f : qdiv(num, delq);
}

// Neighbour values of the gradient and flux arithmetic: read from global memory by
// slot (the phase kernels) or from a tile's shared-memory copy by local id (k_tile).
struct NbGlobal {
  const double* __restrict__ hs;
  const double* __restrict__ z;
  const double* __restrict__ u;
  const double* __restrict__ v;
  const uint8_t* __restrict__ dry;
  __device__ __forceinline__ double H(int i) const { return hs[i]; }
  __device__ __forceinline__ double Z(int i) const { return z[i]; }
  __device__ __forceinline__ double U(int i) const { return u[i]; }
  __device__ __forceinline__ double V(int i) const { return v[i]; }
  __device__ __forceinline__ bool D(int i) const { return dry[i] != 0; }
};
struct NbShared {
  const double *h, *z, *u, *v;
  const uint8_t* dry;
  __device__ __forceinline__ double H(int i) const { return h[i]; }
  __device__ __forceinline__ double Z(int i) const { return z[i]; }
  __device__ __forceinline__ double U(int i) const { return u[i]; }
  __device__ __forceinline__ double V(int i) const { return v[i]; }
  __device__ __forceinline__ bool D(int i) const { return dry[i] != 0; }
};

// Limited LSQ gradients of one cell, with hgradfix2 and the partially-wet velocity
// zeroing (lsq_grad_array.f90:60-73, limiterBJ.f90:42-81 with beta = one,
// cell_grads.f90:72-75, hgradfix2.f90:48-98, to_vertices.f90:44-55).  `c` is the cell
// slot (geometry), `self` its index in `nb`, t3 its face neighbours in `nb` (-1: none)
// and st(k) its k-th stencil neighbour in `nb`.  Differences of the FP64 fields are
// taken in double and then rounded to R.  With the BJ limiter the three rc offsets
// are read here and returned in rcx/rcy (when given).
template <class R>
struct GradOut {
  R hx, hy, ux, uy, vx, vy;
  double ub, vb;
  bool fix;  // hgradfix2 set the gradient: the previous RK level's momentum is zeroed
  bool vz;   // ub, vb are the zeros hgradfix2 / to_vertices set (else the cell's u, v)
};

// The velocity the flux kernels use for cell x this stage (k_grad's ub, vb): FP64,
// the zero hgradfix2 / to_vertices set or the stage-input value, from a flag; mixed,
// the stored value (stored is the velocity array k_grad wrote, d.u_b or d.v_b).
template <class R>
__device__ __forceinline__ double post_fix(const Dev& d, const double* __restrict__ vel,
                                           const double* __restrict__ stored, int x) {
  if (sizeof(R) == 8) return d.vzero[x] ? kZero : vel[x];
  return stored[x];
}

template <class R, class NB, class ST, class VW>
__device__ __forceinline__ GradOut<R> cell_gradients(const Dev& d, const Geo<R>& G, const NB& nb, int c, int self,
                                                     const int (&t3)[3], ST st, VW vwet, R* rcx, R* rcy) {
  const int T = d.T;
  const double zeta_c = nb.H(self) + nb.Z(self);
  const double u_c = nb.U(self), v_c = nb.V(self);
  const bool dry_c = nb.D(self);
  R hx = R(0), hy = R(0), ux = R(0), uy = R(0), vx = R(0), vy = R(0);
  if (d.lim == 1 || d.lim == 2) {
    R dz = R(0), ez = R(0), du = R(0), eu = R(0), dv = R(0), ev = R(0);
    // FP64: lsq_setup's sums over the same stencil values, in its order (used when
    // the layout found them bit-equal to lsq_a/b/c for every cell)
    constexpr bool kF64 = sizeof(R) == 8;
    double sa = 0.0, sb = 0.0, sc = 0.0;
    const int n = d.nst[c];
    int k0 = 0;
    if (n >= 3) {  // interior cells: the three face neighbours, all gathers issued together
      int jj[3];
      R w[3], dx[3], dy[3], pz[3], pu[3], pv[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const int q = k * T + c;
        jj[k] = st(k);
        w[k] = G.st_w[q];
        dx[k] = G.st_dx[q];
        dy[k] = G.st_dy[q];
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        pz[k] = (R)((nb.H(jj[k]) + nb.Z(jj[k])) - zeta_c);
        pu[k] = (R)(nb.U(jj[k]) - u_c);
        pv[k] = (R)(nb.V(jj[k]) - v_c);
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        dz = dz + w[k] * pz[k] * dx[k];
        ez = ez + w[k] * pz[k] * dy[k];
        du = du + w[k] * pu[k] * dx[k];
        eu = eu + w[k] * pu[k] * dy[k];
        dv = dv + w[k] * pv[k] * dx[k];
        ev = ev + w[k] * pv[k] * dy[k];
        if (kF64) {
          sa = sa + (double)w[k] * (double)dx[k] * (double)dx[k];
          sb = sb + (double)w[k] * (double)dx[k] * (double)dy[k];
          sc = sc + (double)w[k] * (double)dy[k] * (double)dy[k];
        }
      }
      k0 = 3;
    }
    for (int k = k0; k < n; k++) {
      const int q = k * T + c;
      const int j = st(k);
      const R w = G.st_w[q], dx = G.st_dx[q], dy = G.st_dy[q];
      const R pz = (R)((nb.H(j) + nb.Z(j)) - zeta_c);
      const R pu = (R)(nb.U(j) - u_c);
      const R pv = (R)(nb.V(j) - v_c);
      dz = dz + w * pz * dx;
      ez = ez + w * pz * dy;
      du = du + w * pu * dx;
      eu = eu + w * pu * dy;
      dv = dv + w * pv * dx;
      ev = ev + w * pv * dy;
      if (kF64) {
        sa = sa + (double)w * (double)dx * (double)dx;
        sb = sb + (double)w * (double)dx * (double)dy;
        sc = sc + (double)w * (double)dy * (double)dy;
      }
    }
    R ai, bi, ci, det;
    if (kF64 && d.lsq_derived) {
      ai = (R)sa;
      bi = (R)sb;
      ci = (R)sc;
      det = (R)(sa * sc - sb * sb);
    } else {
      ai = G.lsq_a[c];
      bi = G.lsq_b[c];
      ci = G.lsq_c[c];
      det = G.lsq_det[c];
    }
    hx = qdiv(ci * dz - bi * ez, det);
    hy = qdiv(ai * ez - dz * bi, det);
    ux = qdiv(ci * du - bi * eu, det);
    uy = qdiv(ai * eu - du * bi, det);
    vx = qdiv(ci * dv - bi * ev, det);
    vy = qdiv(ai * ev - dv * bi, det);
  }
  if (d.lim == 2) {  // limiterBJ.f90:42-81, beta = one
    R rz[3], ru[3], rv[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const int q = j * T + c;
      const int k = t3[j];
      const R rx = G.rc_x[q], ry = G.rc_y[q];
      if (rcx) {
        rcx[j] = rx;
        rcy[j] = ry;
      }
      const double qz = k < 0 ? zeta_c : nb.H(k) + nb.Z(k);
      const double qu = k < 0 ? u_c : nb.U(k);
      const double qv = k < 0 ? v_c : nb.V(k);
      rz[j] = limited_r(zeta_c, qz, hx, hy, rx, ry);
      ru[j] = limited_r(u_c, qu, ux, uy, rx, ry);
      rv[j] = limited_r(v_c, qv, vx, vy, rx, ry);
    }
    const R pz = fmin2(fmin2(rz[0], rz[1]), rz[2]);
    const R pu = fmin2(fmin2(ru[0], ru[1]), ru[2]);
    const R pv = fmin2(fmin2(rv[0], rv[1]), rv[2]);
    hx = pz * hx; hy = pz * hy;
    ux = pu * ux; uy = pu * uy;
    vx = pv * vx; vy = pv * vy;
  }
  hx = hx - G.delz_x[c];
  hy = hy - G.delz_y[c];
  double ub = u_c, vb = v_c;
  bool fix = false, vz = false;
  if (!dry_c) {
    // hgradfix2.f90:48-98
    bool setgrad = zeta_c < d.zmax[c];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const int l = t3[j];
      if (l < 0) continue;
      if (nb.D(l) && nb.Z(l) < zeta_c) setgrad = false;
    }
    if (setgrad) {
      hx = -G.delz_x[c];
      hy = -G.delz_y[c];
      ub = kZero;
      vb = kZero;
      fix = true;
      vz = true;
      ux = R(0); uy = R(0); vx = R(0); vy = R(0);
    }
    // to_vertices.f90:44-55
    bool flag = true;
#pragma unroll
    for (int j = 0; j < 3; j++) flag = flag && vwet(j);
    if (!flag) {
      ub = kZero;
      vb = kZero;
      vz = true;
    }
  }
  GradOut<R> o;
  o.hx = hx; o.hy = hy; o.ux = ux; o.uy = uy; o.vx = vx; o.vy = vy;
  o.ub = ub; o.vb = vb; o.fix = fix; o.vz = vz;
  return o;
}

// Gradients of every cell (list == nullptr) or of the listed cells (the cells with an
// open-boundary face, ahead of the boundary kernel), stored for the phase kernels.
template <class R, bool kList>
__global__ void __launch_bounds__(256, 5) k_grad(Dev d, Geo<R> G, const double* __restrict__ hs,
                                              const uint8_t* __restrict__ dry, double* __restrict__ rku_prev,
                                              double* __restrict__ rkv_prev, const double* __restrict__ u_in,
                                              const double* __restrict__ v_in) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int c;
  if (kList) {
    if (i >= d.nbc_cells) return;
    c = d.bc_cells[i];
  } else {
    if (i >= d.T) return;
    c = i;
  }
  if (!cell_live(d, c)) return;
  const int T = d.T;
  const NbGlobal nb{hs, d.z, u_in, v_in, dry};
  int t3[3];
#pragma unroll
  for (int j = 0; j < 3; j++) t3[j] = d.t2t3[j * T + c];
  const GradOut<R> g = cell_gradients<R>(d, G, nb, c, c, t3, [&](int k) { return d.st_id[k * T + c]; },
                                         [&](int j) { return d.vwet[d.vert[j * T + c]] != 0; },
                                         (R*)nullptr, (R*)nullptr);
  if (g.fix) {
    rku_prev[c] = kZero;
    rkv_prev[c] = kZero;
  }
  G.delh_x[c] = g.hx; G.delh_y[c] = g.hy;
  G.delu_x[c] = g.ux; G.delu_y[c] = g.uy;
  G.delv_x[c] = g.vx; G.delv_y[c] = g.vy;
  if (sizeof(R) == 8) {
    d.vzero[c] = g.vz;
  } else {
    d.u_b[c] = g.ub;
    d.v_b[c] = g.vb;
  }
}

// ---------------------------------------------------------------------------
// Open-boundary fluxes (invisc_fluxes.f90:218-238), one CTA per boundary.  The
// per-edge arithmetic runs on all threads; the sums the reference accumulates
// serially (atotal, newatotal, qtotal, cqin3/cqout3) are added by thread 0 in
// string order, so they round exactly as the reference's loops.
constexpr int kBcThreads = 128;

template <class R>
__global__ void __launch_bounds__(kBcThreads) k_bc(Dev d, Geo<R> G, const double* __restrict__ hs,
                                                   const uint8_t* __restrict__ dry, const double* __restrict__ u_in,
                                                   const double* __restrict__ v_in) {
  const int b = blockIdx.x;
  Scalars* const sc = &d.sc[d.bdr_sid[b]];
  if (sc->converged) return;
  extern __shared__ double smb[];
  const int kind = d.bdr_kind[b], slot = d.bdr_slot[b];
  const int off = d.bdr_off[b], cnt = d.bdr_cnt[b];
  const int T = d.T, NB = d.nbce;
  double* tA = smb;            // [cnt]
  double* tB = smb + cnt;      // [cnt]
  uint8_t* ok = (uint8_t*)(smb + 2 * cnt);
  __shared__ double s_atotal;
  __shared__ int s_done, s_null;
  const double h_dry = d.h_dry;
  // reconstructed edge states (the h/u/v + grad . rc of the boundary element)
  for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
    const int i = d.bce_cell[off + e], m = d.bce_slot[off + e];
    const int q = m * T + i;
    d.bc_rec[off + e] = recon(hs[i], G.delh_x[i], G.rc_x[q], G.delh_y[i], G.rc_y[q]);
    d.bc_rec[NB + off + e] = recon(post_fix<R>(d, u_in, d.u_b, i), G.delu_x[i], G.rc_x[q], G.delu_y[i], G.rc_y[q]);
    d.bc_rec[2 * NB + off + e] = recon(post_fix<R>(d, v_in, d.v_b, i), G.delv_x[i], G.rc_x[q], G.delv_y[i], G.rc_y[q]);
  }
  __syncthreads();
  auto put = [&](int e, double c1, double c2, double c3) {
    d.bc_c[off + e] = c1;
    d.bc_c[NB + off + e] = c2;
    d.bc_c[2 * NB + off + e] = c3;
  };
  if ((kind == BC_QBYH || kind == BC_QBYH_WET) && d.bc_cache) {
    // inflowQbyH.f90:31-212 / :221-402 with the per-edge terms that do not depend on
    // the iterate (edge depth and velocity, the Riemann invariant 2 sqrt(g h) + u.n,
    // normal, length, the wet-only mask) computed once: every fixed-point iteration
    // then evaluates only the qfrac-dependent part, with the same operations in the
    // same order, and thread 0 adds the sums serially in string order.
    const bool wet_only = kind == BC_QBYH_WET;
    const double qin = sc->qin[slot];
    if (qin < kVsmall) {
      for (int e = threadIdx.x; e < cnt; e += blockDim.x) put(e, kZero, kZero, kZero);
      if (threadIdx.x == 0) sc->cqin3[slot] = kZero;
      return;
    }
    double* cb = smb + 2 * cnt;   // [cnt] 2 sqrt(g hleft) + uleft
    double* cnx = cb + cnt;       // [cnt] normal x
    double* cny = cnx + cnt;      // [cnt] normal y
    double* cln = cny + cnt;      // [cnt] edge length
    uint8_t* okc = (uint8_t*)(cln + cnt);  // [cnt] accumulation mask
    uint8_t* v0 = okc + cnt;               // [cnt] wet-only mask
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
      const int i = d.bce_cell[off + e];
      const bool dr = dry[i];
      v0[e] = !(wet_only && dr);
      const double hleft = dr ? kZero : fmax2(d.bc_rec[off + e], kZero);
      tA[e] = hleft * d.bce_len[off + e];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double at = kZero;
      for (int e = 0; e < cnt; e++)
        if (v0[e]) at = at + tA[e];
      s_atotal = at;
      s_null = equals(at, kZero);
      s_done = 0;
    }
    __syncthreads();
    const bool null_area = s_null;
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
      double hleft = null_area ? sc->bch_max : d.bc_rec[off + e], uedg, vedg;
      if (hleft < h_dry) {
        hleft = fmax2(hleft, kZero);
        uedg = kZero;
        vedg = kZero;
      } else {
        uedg = d.bc_rec[NB + off + e];
        vedg = d.bc_rec[2 * NB + off + e];
      }
      const double nx = d.bce_nx[off + e], ny = d.bce_ny[off + e];
      const double uleft = uedg * nx + vedg * ny;
      const double sq = sqrt(kG * hleft);
      cb[e] = 2.0 * sq + uleft;
      cnx[e] = nx;
      cny[e] = ny;
      cln[e] = d.bce_len[off + e];
    }
    __syncthreads();
    // fixed-point iteration on the total flow area (:61-126)
    double newatotal = kZero;
    for (int counter = 0;; counter++) {
      const double atotal = s_atotal;
      const double qfrac = qin / atotal;
      for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
        const double nx = cnx[e], ny = cny[e], len = cln[e];
        double uright = -qfrac;
        double hright = cb[e] - uright;
        hright = hright * hright / 4.0 / kG;
        uright = -qfrac * nx;
        const double vright = -qfrac * ny;
        okc[e] = v0[e] && !(hright < h_dry);
        tA[e] = hright * len;
        tB[e] = (uright * nx + vright * ny) * hright * len;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double na = kZero, qt = kZero;
        int e = 0;
        for (; e + 4 <= cnt; e += 4) {  // loads ahead of the two serial chains
          const uint8_t o0 = okc[e], o1 = okc[e + 1], o2 = okc[e + 2], o3 = okc[e + 3];
          const double a0 = tA[e], a1 = tA[e + 1], a2 = tA[e + 2], a3 = tA[e + 3];
          const double b0 = tB[e], b1 = tB[e + 1], b2 = tB[e + 2], b3 = tB[e + 3];
          if (o0) { na = na + a0; qt = qt + b0; }
          if (o1) { na = na + a1; qt = qt + b1; }
          if (o2) { na = na + a2; qt = qt + b2; }
          if (o3) { na = na + a3; qt = qt + b3; }
        }
        for (; e < cnt; e++)
          if (okc[e]) {
            na = na + tA[e];
            qt = qt + tB[e];
          }
        qt = fabs(qt);
        if (fabs(qt - qin) / qin < 0.005 || counter > 50) s_done = 1;
        else s_atotal = na;
        tA[0] = na;  // hand newatotal to every thread through shared memory
      }
      __syncthreads();
      newatotal = tA[0];
      const int done = s_done;
      __syncthreads();
      if (done) break;
    }
    const double atotal = newatotal;  // :130
    const double qfrac = qin / atotal;
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
      const double nx = cnx[e], ny = cny[e], len = cln[e];
      double uright = -qfrac;
      double hright = cb[e] - uright;
      hright = hright * hright / 4.0 / kG;
      uright = -qfrac * nx;
      const double vright = -qfrac * ny;
      const bool valid = v0[e] && !(hright < h_dry);
      okc[e] = valid;
      if (valid) {
        const double f1 = hright * (uright * nx + vright * ny);
        const double f2 = hright * uright * (uright * nx + vright * ny) + kHalf * kG * hright * hright * nx;
        const double f3 = hright * vright * (uright * nx + vright * ny) + kHalf * kG * hright * hright * ny;
        tA[e] = f1 * len;
        put(e, f1 * len, f2 * len, f3 * len);
      } else {
        put(e, kZero, kZero, kZero);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double cq = kZero;
      for (int e = 0; e < cnt; e++)
        if (okc[e]) cq = cq + tA[e];
      sc->cqin3[slot] = cq;
    }
    return;
  }
  if (kind == BC_QBYH || kind == BC_QBYH_WET) {  // inflowQbyH.f90:31-212 / :221-402
    const bool wet_only = kind == BC_QBYH_WET;
    const double qin = sc->qin[slot];
    if (qin < kVsmall) {
      for (int e = threadIdx.x; e < cnt; e += blockDim.x) put(e, kZero, kZero, kZero);
      if (threadIdx.x == 0) sc->cqin3[slot] = kZero;
      return;
    }
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
      const int i = d.bce_cell[off + e];
      const bool dr = dry[i];
      ok[e] = !(wet_only && dr);
      double hleft = dr ? kZero : fmax2(d.bc_rec[off + e], kZero);
      tA[e] = hleft * d.bce_len[off + e];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double at = kZero;
      for (int e = 0; e < cnt; e++)
        if (ok[e]) at = at + tA[e];
      s_atotal = at;
      s_null = equals(at, kZero);
      s_done = 0;
    }
    __syncthreads();
    const bool null_area = s_null;
    // fixed-point iteration on the total flow area (:61-126)
    double newatotal = kZero;
    for (int counter = 0;; counter++) {
      const double atotal = s_atotal;
      for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
        const int i = d.bce_cell[off + e];
        bool valid = !(wet_only && dry[i]);
        double hleft = null_area ? sc->bch_max : d.bc_rec[off + e], uedg, vedg;
        if (hleft < h_dry) {
          hleft = fmax2(hleft, kZero);
          uedg = kZero;
          vedg = kZero;
        } else {
          uedg = d.bc_rec[NB + off + e];
          vedg = d.bc_rec[2 * NB + off + e];
        }
        const double nx = d.bce_nx[off + e], ny = d.bce_ny[off + e], len = d.bce_len[off + e];
        const double qfrac = qin / atotal;
        double uright = -qfrac;
        const double uleft = uedg * nx + vedg * ny;
        const double sq = sqrt(kG * hleft);
        double hright = 2.0 * sq + uleft - uright;
        hright = hright * hright / 4.0 / kG;
        uright = -qfrac * nx;
        const double vright = -qfrac * ny;
        if (hright < h_dry) valid = false;
        ok[e] = valid;
        tA[e] = hright * len;
        tB[e] = (uright * nx + vright * ny) * hright * len;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double na = kZero, qt = kZero;
        for (int e = 0; e < cnt; e++)
          if (ok[e]) {
            na = na + tA[e];
            qt = qt + tB[e];
          }
        qt = fabs(qt);
        if (fabs(qt - qin) / qin < 0.005 || counter > 50) s_done = 1;
        else s_atotal = na;
        tA[0] = na;  // hand newatotal to every thread through shared memory
      }
      __syncthreads();
      newatotal = tA[0];
      const int done = s_done;
      __syncthreads();
      if (done) break;
    }
    const double atotal = newatotal;  // :130
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
      const int i = d.bce_cell[off + e];
      bool valid = !(wet_only && dry[i]);
      double hleft = null_area ? sc->bch_max : d.bc_rec[off + e], uedg, vedg;
      if (hleft < h_dry) {
        hleft = fmax2(hleft, kZero);
        uedg = kZero;
        vedg = kZero;
      } else {
        uedg = d.bc_rec[NB + off + e];
        vedg = d.bc_rec[2 * NB + off + e];
      }
      const double nx = d.bce_nx[off + e], ny = d.bce_ny[off + e], len = d.bce_len[off + e];
      const double qfrac = qin / atotal;
      double uright = -qfrac;
      const double uleft = uedg * nx + vedg * ny;
      const double sq = sqrt(kG * hleft);
      double hright = 2.0 * sq + uleft - uright;
      hright = hright * hright / 4.0 / kG;
      uright = -qfrac * nx;
      const double vright = -qfrac * ny;
      if (hright < h_dry) valid = false;
      ok[e] = valid;
      if (valid) {
        const double f1 = hright * (uright * nx + vright * ny);
        const double f2 = hright * uright * (uright * nx + vright * ny) + kHalf * kG * hright * hright * nx;
        const double f3 = hright * vright * (uright * nx + vright * ny) + kHalf * kG * hright * hright * ny;
        tA[e] = f1 * len;
        put(e, f1 * len, f2 * len, f3 * len);
      } else {
        put(e, kZero, kZero, kZero);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double cq = kZero;
      for (int e = 0; e < cnt; e++)
        if (ok[e]) cq = cq + tA[e];
      sc->cqin3[slot] = cq;
    }
    return;
  }
  // The remaining routines have no cross-edge coupling.
  for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
    const int i = d.bce_cell[off + e];
    const bool dr = dry[i];
    const double nx = d.bce_nx[off + e], ny = d.bce_ny[off + e];
    const double tx = d.bce_tx[off + e], ty = d.bce_ty[off + e];
    const double len = d.bce_len[off + e], zmid = d.bce_zmid[off + e];
    double hleft = d.bc_rec[off + e];
    const double ur0 = d.bc_rec[NB + off + e], vr0 = d.bc_rec[2 * NB + off + e];
    double f[3] = {kZero, kZero, kZero};
    bool valid = true;
    if (kind == BC_HIN) {  // inflowH.f90:28-93
      double uedg, vedg;
      hleft = fmax2(hleft, kZero);
      if (hs[i] < h_dry) { uedg = kZero; vedg = kZero; }
      else { uedg = ur0; vedg = vr0; }
      const double hright = fmax2(kZero, sc->qin[slot] - zmid);
      double uleft = uedg * nx + vedg * ny;
      const double sl = sqrt(kG * hleft), sr = sqrt(kG * hright);
      double uright = uleft + (sl - sr);
      const double vright = uright * ny;
      uright = uright * nx;
      uleft = uedg;
      const double vleft = vedg;
      if (hleft < h_dry && hright < h_dry) valid = false;
      else flux_roe<double>(nx, ny, hleft, uleft, vleft, hright, uright, vright, f);
      if (valid) { tA[e] = f[0] * len; put(e, f[0] * len, f[1] * len, f[2] * len); }
    } else if (kind == BC_HOUT) {  // outflowbyH.f90:30-137
      double uedg, vedg;
      if (dr || hleft < h_dry) { uedg = kZero; vedg = kZero; hleft = fmax2(hleft, kZero); }
      else { uedg = ur0; vedg = vr0; }
      double hright = fmax2(kZero, sc->hbc[slot] - zmid);
      if (hleft < h_dry && hright < h_dry) valid = false;
      else {
        double uleft, vleft, uright, vright;
        if (hright < h_dry) {
          uright = kZero; uleft = uedg; vright = kZero; vleft = vedg;
        } else {
          uleft = uedg * nx + vedg * ny;
          vleft = uedg * tx + vedg * ty;
          const double sl = sqrt(kG * hleft), sr = sqrt(kG * hright);
          uright = uleft + (sl - sr);
          vright = vleft;
          uleft = uedg;
          vleft = vedg;
          uedg = uright;
          vedg = vright;
          uright = uedg * nx + vedg * tx;
          vright = uedg * ny + vedg * ty;
        }
        bool set_wall = false;
        if (d.hvalve) {
          const double dot = uright * nx + vright * ny;
          if (dot < kZero) { set_wall = true; hright = hleft; uright = kZero; vright = kZero; }
        }
        flux_roe<double>(nx, ny, hleft, uleft, vleft, hright, uright, vright, f);
        if (set_wall) f[0] = kZero;
        tA[e] = f[0] * len;
        put(e, f[0] * len, f[1] * len, f[2] * len);
      }
    } else if (kind == BC_CRIT) {  // crit_outflow.f90:29-107
      double uedg, vedg;
      if (dr || hleft < h_dry) { uedg = kZero; vedg = kZero; hleft = fmax2(hleft, kZero); }
      else { uedg = ur0; vedg = vr0; }
      if (hleft < h_dry) valid = false;
      else {
        const double uleft = uedg * nx + vedg * ny;
        const double vleft = uedg * tx + vedg * ty;
        double uright = uleft, vright = vleft;
        double hright = uright * uright / kG;
        uedg = uright;
        vedg = vright;
        uright = uedg * nx + vedg * tx;
        vright = uedg * ny + vedg * ty;
        if (d.hvalve) {
          const double dot = uright * nx + vright * ny;
          if (dot < kZero) { hright = hleft; uright = kZero; vright = kZero; }
        }
        f[0] = hright * (uright * nx + vright * ny);
        f[1] = hright * uright * (uright * nx + vright * ny) + kHalf * kG * hright * hright * nx;
        f[2] = hright * vright * (uright * nx + vright * ny) + kHalf * kG * hright * hright * ny;
        const double dh = kZero;  // :97-99
        tA[e] = f[0] * len;
        put(e, f[0] * len, (f[1] + dh * nx) * len, (f[2] + dh * ny) * len);
      }
    } else {  // BC_FREE, free_flow.f90:30-93
      double uedg, vedg;
      hleft = fmax2(hleft, kZero);
      if (hleft < h_dry) valid = false;
      else {
        if (hs[i] < h_dry) { uedg = kZero; vedg = kZero; }
        else { uedg = ur0; vedg = vr0; }
        const double uleft = uedg, vleft = vedg;
        double hright = hleft, uright = uleft, vright = vleft;
        bool set_wall = false;
        if (d.hvalve) {
          const double dot = uright * nx + vright * ny;
          if (dot < 0) { set_wall = true; uright = kZero; vright = kZero; }
        }
        flux_roe<double>(nx, ny, hleft, uleft, vleft, hright, uright, vright, f);
        if (set_wall) f[0] = kZero;
        put(e, f[0] * len, f[1] * len, f[2] * len);
      }
    }
    ok[e] = valid;
    if (!valid) put(e, kZero, kZero, kZero);
  }
  __syncthreads();
  if (threadIdx.x == 0 && kind != BC_FREE) {
    double cq = kZero;
    for (int e = 0; e < cnt; e++)
      if (ok[e]) cq = cq + tA[e];
    if (kind == BC_HIN) sc->cqin3[slot] = cq;
    else sc->cqout3[slot] = cq;
  }
}

// ---------------------------------------------------------------------------
// Reconstructed edge state of cell x at its local slot m (invisc_fluxes.f90:53-81).
struct EdgeState {
  double h, u, v;
};

template <class R>
__device__ __forceinline__ EdgeState edge_state(const Dev& d, const Geo<R>& G, const double* __restrict__ hs,
                                                const double* __restrict__ u_in, const double* __restrict__ v_in,
                                                int x, int m) {
  const int q = m * d.T + x;
  const R rx = G.rc_x[q], ry = G.rc_y[q];
  EdgeState s;
  s.h = recon(hs[x], G.delh_x[x], rx, G.delh_y[x], ry);
  if (s.h < kZero) s.h = kZero;
  s.u = recon(post_fix<R>(d, u_in, d.u_b, x), G.delu_x[x], rx, G.delu_y[x], ry);
  s.v = recon(post_fix<R>(d, v_in, d.v_b, x), G.delv_x[x], rx, G.delv_y[x], ry);
  return s;
}

// invisc_fluxes.f90:39-147 for an interior edge from its two face states: left =
// e(1), right = e(2), dl/dr their dry flags, zl/zr their bed elevations and hl/hr
// their cell depths (Rusanov's cell celerities); returns false when the edge is
// skipped.  The wet/dry tests and the I1 stage comparison run on the FP64 face
// states; the flux function in R.
template <class R>
__device__ __forceinline__ bool edge_flux(const Dev& d, bool dl, bool dr, const EdgeState& sl, const EdgeState& sr,
                                          double zl, double zr, double hl, double hr, R nx, R ny, double z0e, R* f,
                                          bool* bad) {
  if (dl && dr) return false;
  double hleft = kZero, uleft = kZero, vleft = kZero, hright = kZero, uright = kZero, vright = kZero;
  if (!dl) {
    hleft = sl.h; uleft = sl.u; vleft = sl.v;
  }
  if (!dr) {
    hright = sr.h; uright = sr.u; vright = sr.v;
  }
  if (hleft < d.h_dry && hright < d.h_dry) return false;
  bool set_wall = false;
  if (dl || dr) {  // ALGORITHM I1
    double h0 = fmax2(hright, hleft);
    h0 = h0 + z0e;
    if (dl)
      if (zl + d.h_wet > h0) { set_wall = true; hleft = hright; }
    if (dr)
      if (zr + d.h_wet > h0) { set_wall = true; hright = hleft; }
  }
  if (set_wall) {
    f[0] = R(kZero);
    const R hw = (R)fmax2(hleft, hright);
    f[1] = R(kHalf) * R(kG) * hw * hw * nx;
    f[2] = R(kHalf) * R(kG) * hw * hw * ny;
  } else if (d.flux == STORM_FLUX_HLL) {
    flux_hll<R>(nx, ny, (R)hleft, (R)uleft, (R)vleft, (R)hright, (R)uright, (R)vright, (R)d.h_dry, f, bad);
  } else if (d.flux == STORM_FLUX_RUSANOV) {
    const R cl = dl ? R(kZero) : (R)sqrt(kG * hl);  // wavec (solverFVT.f90:180-181)
    const R cr = dr ? R(kZero) : (R)sqrt(kG * hr);
    flux_rusanov<R>(nx, ny, (R)hleft, (R)uleft, (R)vleft, cl, (R)hright, (R)uright, (R)vright, cr, f);
  } else {
    flux_roe<R>(nx, ny, (R)hleft, (R)uleft, (R)vleft, (R)hright, (R)uright, (R)vright, f);
  }
  return true;
}

// The same for the edge between L=e(1) (slot ml) and R=e(2) (slot mr), with the face
// states reconstructed from the stored gradients.
template <class R>
__device__ __forceinline__ bool interior_flux(const Dev& d, const Geo<R>& G, const double* __restrict__ hs,
                                              const uint8_t* __restrict__ dry, const double* __restrict__ u_in,
                                              const double* __restrict__ v_in, int L, int ml, int Rc, int mr, R nx,
                                              R ny, double z0e, R* f, bool* bad) {
  const bool dl = dry[L], dr = dry[Rc];
  if (dl && dr) return false;
  EdgeState sl{kZero, kZero, kZero}, sr{kZero, kZero, kZero};
  if (!dl) sl = edge_state(d, G, hs, u_in, v_in, L, ml);
  if (!dr) sr = edge_state(d, G, hs, u_in, v_in, Rc, mr);
  return edge_flux<R>(d, dl, dr, sl, sr, d.z[L], d.z[Rc], hs[L], hs[Rc], nx, ny, z0e, f, bad);
}

// Interior-edge fluxes of one stage (invisc_fluxes.f90:39-147), one thread per edge:
// the flux of edge k is evaluated once, in the reference's orientation (left =
// edges(k)%e(1)), and stored as f*length, the amount the reference subtracts from
// phi(e(1),:) and adds to phi(e(2),:).
template <class R>
__global__ void __launch_bounds__(128, 8) k_eflux(Dev d, Geo<R> G, const double* __restrict__ hs,
                                               const uint8_t* __restrict__ dry, const double* __restrict__ u_in,
                                               const double* __restrict__ v_in) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.ne) return;
  if (!item_live(d, d.edge_sid, e)) return;
  const int L = d.eL[e], Rc = d.eR[e];
  const uint8_t sl = d.eslot[e];
  R f[3];
  bool bad = false;
  const bool ok = interior_flux<R>(d, G, hs, dry, u_in, v_in, L, sl & 3, Rc, (sl >> 2) & 3, G.enx[e], G.eny[e],
                                   (dry[L] || dry[Rc]) ? d.ez0[e] : kZero, f, &bad);
  d.eok[e] = ok;
  if (ok) {
    const R len = G.elen[e];
    G.efx[e] = f[0] * len;
    G.efx[d.ne + e] = f[1] * len;
    G.efx[2 * d.ne + e] = f[2] * len;
  }
  if (bad) atomicOr(&d.sc[d.edge_sid[e]].status, 2);
}

// bed_slope_STD.f90:23-70 with adjustZb.f90:41-70: the amounts g*h*gradzb*area that
// are subtracted from phi(i,2:3), from the cell's depth gradient (dhx, dhy).  The
// vertex offsets from the centroid (node - centroid, the reference's own differences)
// are precomputed per cell; the adjust test (a negative reconstructed vertex depth)
// and the adjusted gradient run in double on both paths.
__device__ __forceinline__ void bed_source(const Dev& d, const Geo<double>& G, int c, double h_c, double dhx,
                                           double dhy, double* s2, double* s3) {
  const int T = d.T;
  double hp[3];
  bool adjust = false;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const int q = i * T + c;
    hp[i] = h_c + dhx * d.vox[q] + dhy * d.voy[q];
    if (hp[i] < kZero) adjust = true;
  }
  double gx, gy;
  if (adjust) {
    double zp[3], x[3], y[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int vid = d.vert[i * T + c];
      hp[i] = fmin2(kZero, hp[i]);
      zp[i] = d.zvtx[vid] + hp[i];
      x[i] = d.node_x[vid];
      y[i] = d.node_y[vid];
    }
    const double b1 = y[1] - y[2], c1 = x[2] - x[1];
    const double b2 = y[2] - y[0], c2 = x[0] - x[2];
    const double b3 = y[0] - y[1], c3 = x[1] - x[0];
    const double a = kHalf / d.area[c];
    gx = a * (b1 * zp[0] + b2 * zp[1] + b3 * zp[2]);
    gy = a * (c1 * zp[0] + c2 * zp[1] + c3 * zp[2]);
  } else {
    gx = G.delz_x[c];
    gy = G.delz_y[c];
  }
  *s2 = kG * h_c * gx * d.area[c];
  *s3 = kG * h_c * gy * d.area[c];
}
__device__ __forceinline__ void bed_source(const Dev& d, const Geo<float>& G, int c, double h_c, float dhx,
                                           float dhy, double* s2, double* s3) {
  const int T = d.T;
  double hp[3];
  bool adjust = false;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const int q = i * T + c;
    hp[i] = h_c + (double)(dhx * G.vox[q] + dhy * G.voy[q]);
    if (hp[i] < kZero) adjust = true;
  }
  if (adjust) {
    double zp[3], x[3], y[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int vid = d.vert[i * T + c];
      zp[i] = d.zvtx[vid] + fmin2(kZero, hp[i]);
      x[i] = d.node_x[vid];
      y[i] = d.node_y[vid];
    }
    const double a = kHalf / d.area[c];
    const double gx = a * ((y[1] - y[2]) * zp[0] + (y[2] - y[0]) * zp[1] + (y[0] - y[1]) * zp[2]);
    const double gy = a * ((x[2] - x[1]) * zp[0] + (x[0] - x[2]) * zp[1] + (x[1] - x[0]) * zp[2]);
    *s2 = kG * h_c * gx * d.area[c];
    *s3 = kG * h_c * gy * d.area[c];
  } else {
    const float ga = 9.81f * (float)h_c * (float)d.area[c];
    *s2 = (double)(ga * G.delz_x[c]);
    *s3 = (double)(ga * G.delz_y[c]);
  }
}

// Where the face contributions of a cell come from: the phase kernels' global arrays
// (edge fluxes of k_eflux, stored gradients) ...
template <class R>
struct FacesGlobal {
  const Dev& d;
  const Geo<R>& G;
  const double* __restrict__ hs;
  int c;
  const double* __restrict__ u_in;  // stage-input velocities (the cell's own, for weslp2 walls)
  const double* __restrict__ v_in;
  // the faces in the order their terms are added (slots, kinds, references), read
  // from the per-cell arrays kept in that order so that none waits on forder
  __device__ __forceinline__ uint8_t order(int (&fj)[3], int (&fkd)[3], int (&fe)[3]) const {
    const uint8_t ord = d.forder[c];
    const unsigned ko = d.fko[c];
#pragma unroll
    for (int t = 0; t < 3; t++) {
      fj[t] = (ord >> (2 * t)) & 3;
      fkd[t] = (ko >> (3 * t)) & 7;
      fe[t] = d.frefo[t * d.T + c];
    }
    return ord;
  }
  // flux*length of the interior face in slot j (edge e), and whether the edge produced one
  __device__ __forceinline__ bool iface(int j, int e, R* f) const {
    f[0] = G.efx[e];
    f[1] = G.efx[d.ne + e];
    f[2] = G.efx[2 * d.ne + e];
    return d.eok[e] != 0;
  }
  // the cell's own reconstructed state at face j (weslp2 walls)
  __device__ __forceinline__ EdgeState own(int j) const {
    const int q = j * d.T + c;
    EdgeState s;
    s.h = recon(hs[c], G.delh_x[c], G.rc_x[q], G.delh_y[c], G.rc_y[q]);
    s.u = recon(post_fix<R>(d, u_in, d.u_b, c), G.delu_x[c], G.rc_x[q], G.delu_y[c], G.rc_y[q]);
    s.v = recon(post_fix<R>(d, v_in, d.v_b, c), G.delv_x[c], G.rc_x[q], G.delv_y[c], G.rc_y[q]);
    return s;
  }
  __device__ __forceinline__ void dh(R* x, R* y) const {
    *x = G.delh_x[c];
    *y = G.delh_y[c];
  }
  // vertex depths at the two ends (walledg1 order) of the wall face in slot j (wall w)
  __device__ __forceinline__ void hwall(int j, int w, double* h1, double* h2) const {
    *h1 = d.hvtx[d.wall_p1[w]];
    *h2 = d.hvtx[d.wall_p2[w]];
  }
};

// ... or a tile's shared memory (k_tile): edge fluxes by local edge, face states and
// depth gradients by local cell.
template <class R>
struct FacesTile {
  const uint16_t* __restrict__ lfe;
  int T, c, l, ngm, nem;
  const R* sf;             // [3][nem]
  const uint8_t* seok;     // [nem]
  const double *sfh, *sfu, *sfv;  // [3][ngm]
  const R *sdhx, *sdhy;    // [owned]
  const uint32_t* __restrict__ lwall;  // [3][T] local node ids of the wall ends
  const double* shv;       // vertex depths of the tile's nodes
  const double* __restrict__ hvtx;  // or the global ones (nodes not fused)
  const int32_t* __restrict__ wall_p1;
  const int32_t* __restrict__ wall_p2;
  const int32_t* __restrict__ fref;
  const uint8_t* __restrict__ forder;
  const uint8_t* __restrict__ fkind;
  __device__ __forceinline__ uint8_t order(int (&fj)[3], int (&fkd)[3], int (&fe)[3]) const {
    const uint8_t ord = forder[c];
#pragma unroll
    for (int t = 0; t < 3; t++) {
      fj[t] = (ord >> (2 * t)) & 3;
      fkd[t] = fkind[fj[t] * T + c] & 7;
      fe[t] = fref[fj[t] * T + c];
    }
    return ord;
  }
  __device__ __forceinline__ void hwall(int j, int w, double* h1, double* h2) const {
    if (shv) {
      const uint32_t lw = lwall[j * T + c];
      *h1 = shv[lw & 0xFFFF];
      *h2 = shv[lw >> 16];
    } else {
      *h1 = hvtx[wall_p1[w]];
      *h2 = hvtx[wall_p2[w]];
    }
  }
  __device__ __forceinline__ bool iface(int j, int, R* f) const {
    const int le = lfe[j * T + c];
    f[0] = sf[le];
    f[1] = sf[nem + le];
    f[2] = sf[2 * nem + le];
    return seok[le] != 0;
  }
  // the face state is clipped at zero depth; weslp2 skips any face state below
  // h_dry > 0, so the clip never changes its result
  __device__ __forceinline__ EdgeState own(int j) const {
    EdgeState s;
    s.h = sfh[j * ngm + l];
    s.u = sfu[j * ngm + l];
    s.v = sfv[j * ngm + l];
    return s;
  }
  __device__ __forceinline__ void dh(R* x, R* y) const {
    *x = sdhx[l];
    *y = sdhy[l];
  }
};

// Fluxes and sources of stage s for cell c: the faces are added to phi in the order
// invisc_fluxes.f90 visits them (phi = zero first, solverFVT.f90:194), then the bed
// slope, wind and culvert terms.  phi is FP64 on both paths.
template <class R, class FS>
__device__ __forceinline__ void assemble_phi(const Dev& d, const Geo<R>& G, const FS& fs, int c, double h_c,
                                             bool dry_c, double* p1o, double* p2o, double* p3o) {
  const int T = d.T;
  double p1 = kZero, p2 = kZero, p3 = kZero;
  // Issue the loads of all three faces before the (ordered) accumulation: face
  // descriptors first, then the fluxes of the interior faces, so the gathers overlap
  // instead of forming one dependent chain per face.
  int fj[3], fkd[3], fe[3];
  const uint8_t ord = fs.order(fj, fkd, fe);
  bool fok[3];
  R fv[3][3];
#pragma unroll
  for (int t = 0; t < 3; t++) {
    fok[t] = false;
    fv[t][0] = fv[t][1] = fv[t][2] = R(0);
    if (fkd[t] == FACE_LEFT || fkd[t] == FACE_RIGHT) fok[t] = fs.iface(fj[t], fe[t], fv[t]);
  }
#pragma unroll
  for (int t = 0; t < 3; t++) {
    const int j = fj[t];
    const int q = j * T + c;
    const int kind = fkd[t];
    if (kind == FACE_LEFT || kind == FACE_RIGHT) {
      if (fok[t]) {
        const double f0 = fv[t][0], f1 = fv[t][1], f2 = fv[t][2];
        if (kind == FACE_LEFT) {
          p1 = p1 - f0;
          p2 = p2 - f1;
          p3 = p3 - f2;
        } else {
          p1 = p1 + f0;
          p2 = p2 + f1;
          p3 = p3 + f2;
        }
      }
    } else if (kind == FACE_WALL) {
      if (dry_c) continue;
      const double nx = d.fnx[q], ny = d.fny[q], len = d.flen[q];
      if (d.btype == 0) {  // wenslp3_fluxes.f90:34-67
        double h1, h2;
        fs.hwall(j, fe[t], &h1, &h2);
        double hedge = qsqrt((h1 * h1 + h1 * h2 + h2 * h2) * kOneThird);
        if (hedge < kZero) hedge = kZero;
        if (hedge < d.h_dry) continue;
        p2 = p2 - kHalf * kG * hedge * hedge * nx * len;
        p3 = p3 - kHalf * kG * hedge * hedge * ny * len;
      } else {  // weslp2_fluxes.f90:34-76
        const EdgeState o = fs.own(j);
        const double hleft = o.h;
        if (hleft < d.h_dry) continue;
        const double uleft = o.u;
        const double vleft = o.v;
        const double tx = -ny, ty = nx;  // edges%tang flipped with the normal
        double uright = uleft * tx + vleft * ty;
        uright = uright + 2.0 * sqrt(kG * hleft);
        const double hright = uright * uright / 4.0 / kG;
        const double f2 = kHalf * kG * hright * hright * nx;
        const double f3 = kHalf * kG * hright * hright * ny;
        const double dh = kZero;
        p2 = p2 - (f2 + dh * nx) * len;
        p3 = p3 - (f3 + dh * ny) * len;
      }
    } else if (kind == FACE_BC) {
      const int e = fe[t];
      p1 = p1 - d.bc_c[e];
      p2 = p2 - d.bc_c[d.nbce + e];
      p3 = p3 - d.bc_c[2 * d.nbce + e];
    }
  }
  if (!dry_c) {
    double s2, s3;
    R dhx, dhy;
    fs.dh(&dhx, &dhy);
    bed_source(d, G, c, h_c, dhx, dhy, &s2, &s3);
    p2 = p2 - s2;
    p3 = p3 - s3;
    if (d.wcoef1) {  // wind forcing (solverFVT.f90:218-224)
      p2 = p2 + d.wcoef1[c];
      p3 = p3 + d.wcoef2[c];
    }
  }
  if (ord & kOrderHasCulvert) {  // culvert sources and sinks (solverFVT.f90:227-233)
    int lo = 0, hi = d.ncvc;  // first term of cell c
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (d.cvc_cell[mid] < c) lo = mid + 1;
      else hi = mid;
    }
    for (int k = lo; k < d.ncvc && d.cvc_cell[k] == c; k++) {
      const int code = d.cvc_code[k];
      if (code & 1) p1 = p1 + d.cvsrc[code >> 1];
      else p1 = p1 - d.cvsrc[code >> 1];
    }
  }
  *p1o = p1;
  *p2o = p2;
  *p3o = p3;
}

// The RK update of stage s (1-based) for cell c from its phi (solverFVT.f90:259-325).
__device__ __forceinline__ void rk_update(const Dev& d, int s, int c, double h_c, bool dry_c, double p1, double p2,
                                          double p3, uint8_t* __restrict__ dry_next, const double* __restrict__ u_in,
                                          const double* __restrict__ v_in, double* __restrict__ u_out,
                                          double* __restrict__ v_out) {
  const int T = d.T;
  // RK update (solverFVT.f90:259-283)
  const double u_c = u_in[c], v_c = v_in[c];
  double delt;
  if (d.steady) {
    const double um = (h_c < d.h_dry) ? kZero : qsqrt(u_c * u_c + v_c * v_c);
    const double wc = dry_c ? kZero : sqrt(kG * h_c);
    delt = um + wc;
    if (delt < SMALL_F) delt = 1.044;
    delt = d.cfl * d.area[c] / (delt * d.perim[c]);
    Scalars& sc = d.sc[cell_scenario(d, c)];
    if (s == d.K && c == sc.last_cell) sc.delt_fric = delt;
  } else {
    delt = d.sc[cell_scenario(d, c)].delt;
  }
  const double dt = delt / d.area[c];
  double rh = kZero, ru = kZero, rv = kZero;
  for (int j = 0; j <= s - 1; j++) {
    // a zero coefficient (SSP-RK3 stage 3, level 1) adds a signed zero to a sum that
    // started at +0, which leaves its bits unchanged: skip the loads
    if (d.alpha[s][j] == kZero) continue;
    const int q = j * T + c;
    rh = rh + d.alpha[s][j] * d.rkh[q];
    ru = ru + d.alpha[s][j] * d.rku[q];
    rv = rv + d.alpha[s][j] * d.rkv[q];
  }
  rh = rh + d.beta[s] * dt * p1;
  ru = (ru + d.beta[s] * dt * p2);
  rv = (rv + d.beta[s] * dt * p3);
  if (d.vclip) {  // :286-296
    const double heff = fmax2(d.h_dry, rh);
    const double umag = sqrt(ru * ru + rv * rv) / heff;
    if (umag > d.vceiling) {
      ru = d.vceiling * ru / umag;
      rv = d.vceiling * rv / umag;
    }
  }
  rh = fmax2(rh, kZero);  // :300-325
  double un, vn;
  const double h_delta = dry_c ? d.h_wet : d.h_dry;
  if (rh > h_delta) {
    un = qdiv(ru, rh);
    vn = qdiv(rv, rh);
  } else {
    ru = kZero; rv = kZero; un = kZero; vn = kZero;
  }
  const int qs = s * T + c;
  d.rkh[qs] = rh;
  d.rku[qs] = ru;
  d.rkv[qs] = rv;
  u_out[c] = un;
  v_out[c] = vn;
  if (s < d.K) {
    double um;
    dry_next[c] = dry_flag(rh, un, vn, d.h_dry, d.h_wet, &um);
  } else {
    d.phimax[c] = fmax2(fmax2(fmax2(kZero, fabs(p1)), fabs(p2)), fabs(p3));
  }
}

template <class R>
__device__ __forceinline__ void flux_cell(const Dev& d, const Geo<R>& G, int s, int c, const double* __restrict__ hs,
                                          const uint8_t* __restrict__ dry, uint8_t* __restrict__ dry_next,
                                          const double* __restrict__ u_in, const double* __restrict__ v_in,
                                          double* __restrict__ u_out, double* __restrict__ v_out) {
  double p1, p2, p3;
  const double h_c = hs[c];
  const bool dry_c = dry[c] != 0;
  assemble_phi<R>(d, G, FacesGlobal<R>{d, G, hs, c, u_in, v_in}, c, h_c, dry_c, &p1, &p2, &p3);
  rk_update(d, s, c, h_c, dry_c, p1, p2, p3, dry_next, u_in, v_in, u_out, v_out);
}

// Residual smoothing (solverFVT.f90:238-256, activateRSAVG): the stage's phi is
// assembled into d.phi (and its copy phi0), smoothed by Gauss-Seidel passes over the
// cells of one colour of the t2t stencil at a time (cells of a colour share no
// stencil edge, so each reads its neighbours' latest values exactly as a serial sweep
// in colour order does), then every cell is updated.
template <class R>
__global__ void __launch_bounds__(128) k_flux_phi(Dev d, Geo<R> G, const double* __restrict__ hs,
                                              const uint8_t* __restrict__ dry, const double* __restrict__ u_in,
                                              const double* __restrict__ v_in, int bc_cells) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int c;
  if (bc_cells) {
    if (i >= d.nbc_cells) return;
    c = d.bc_cells[i];
  } else {
    if (i >= d.T) return;
    c = i;
    if (d.forder[c] & kOrderHasBc) return;
  }
  if (!cell_live(d, c)) return;
  double p1, p2, p3;
  assemble_phi<R>(d, G, FacesGlobal<R>{d, G, hs, c, u_in, v_in}, c, hs[c], dry[c] != 0, &p1, &p2, &p3);
  const size_t T = d.T;
  d.phi[c] = p1;
  d.phi[T + c] = p2;
  d.phi[2 * T + c] = p3;
  d.phi0[c] = p1;
  d.phi0[T + c] = p2;
  d.phi0[2 * T + c] = p3;
}

#ifndef STORM_FVT_F32_TU
__global__ void __launch_bounds__(256) k_rsavg(Dev d, int off, int cnt) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= cnt) return;
  const int c = d.rs_cells[off + q];
  if (!cell_live(d, c)) return;
  const size_t T = d.T;
  const int n = d.nst[c];
  for (int k = 0; k < 3; k++) {
    double p = d.rs_fac1 * d.phi0[k * T + c];
    for (int m = 0; m < n; m++) p = p + d.rs_fac2 * d.phi[k * T + d.st_id[m * T + c]];
    d.phi[k * T + c] = p;
  }
}

__global__ void __launch_bounds__(128) k_update(Dev d, int s, const double* __restrict__ hs,
                                            const uint8_t* __restrict__ dry, uint8_t* __restrict__ dry_next) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.T) return;
  if (!cell_live(d, c)) return;
  const size_t T = d.T;
  rk_update(d, s, c, hs[c], dry[c] != 0, d.phi[c], d.phi[T + c], d.phi[2 * T + c], dry_next, d.u_a, d.v_a, d.u_a,
            d.v_a);
}
#endif  // !STORM_FVT_F32_TU

// All cells without an open-boundary face (those wait for k_bc in k_flux_bc).
template <class R>
__global__ void __launch_bounds__(128, 10) k_flux(Dev d, Geo<R> G, int s, const double* __restrict__ hs,
                                              const uint8_t* __restrict__ dry, uint8_t* __restrict__ dry_next,
                                              const double* __restrict__ u_in, const double* __restrict__ v_in,
                                              double* __restrict__ u_out, double* __restrict__ v_out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.T) return;
  if (!cell_live(d, c)) return;
  if (d.forder[c] & kOrderHasBc) return;
  flux_cell<R>(d, G, s, c, hs, dry, dry_next, u_in, v_in, u_out, v_out);
}

// The cells with an open-boundary face, after k_bc.
template <class R>
__global__ void __launch_bounds__(128) k_flux_bc(Dev d, Geo<R> G, int s, const double* __restrict__ hs,
                                                 const uint8_t* __restrict__ dry, uint8_t* __restrict__ dry_next,
                                                 const double* __restrict__ u_in, const double* __restrict__ v_in,
                                                 double* __restrict__ u_out, double* __restrict__ v_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.nbc_cells) return;
  const int c = d.bc_cells[i];
  if (!cell_live(d, c)) return;
  flux_cell<R>(d, G, s, c, hs, dry, dry_next, u_in, v_in, u_out, v_out);
}

// ---------------------------------------------------------------------------
// The fused RK stage over Morton tiles (one CTA per tile of kTileCells cell slots):
//   A  the stage-input state (h, z, u, v, dry flag) of the tile's owned, H1 and H2
//      cells into shared memory (owned cells: coalesced; halo: gathered);
//   B  gradients, limiter, hgradfix2 and velocity zeroing of the owned and H1 cells
//      (cell_gradients, the phase kernels' arithmetic) and their three face states;
//   C  the flux of every edge of an owned cell, once, in the reference's orientation
//      (edge_flux); the fluxes the boundary cells' update needs go to global memory;
//   D  the ordered face gather, sources and SSP-RK update of every owned cell
//      without an open-boundary face (assemble_phi + rk_update).
// The boundary cells keep the phase path: their gradients (k_grad over the
// boundary-cell list) and k_bc run on the side stream beside this kernel, and
// k_flux_bc updates them afterwards.  Velocities ping-pong between two buffers: a
// tile may still read a neighbour's stage-input velocity while the neighbour's own
// tile writes its new one.
constexpr int kTileThreads = 256;  // tiles of 256 cell slots (the host's tile plan)

struct TileSmem {
  size_t h, z, u, v, fh, fu, fv, dhx, dhy, f, hv, dry, eok, vw, total;
};
__host__ __device__ inline TileSmem tile_smem_layout(int ns, int ng, int ne, int tc, int rsz, int nn) {
  TileSmem m;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t r = o;
    o += (bytes + 15) & ~(size_t)15;
    return r;
  };
  m.h = take(8 * (size_t)ns);
  m.z = take(8 * (size_t)ns);
  m.u = take(8 * (size_t)ns);
  m.v = take(8 * (size_t)ns);
  m.fh = take(8 * 3 * (size_t)ng);
  m.fu = take(8 * 3 * (size_t)ng);
  m.fv = take(8 * 3 * (size_t)ng);
  m.dhx = take((size_t)rsz * tc);
  m.dhy = take((size_t)rsz * tc);
  m.f = take((size_t)rsz * 3 * ne);
  m.hv = take(8 * (size_t)nn);
  m.dry = take(ns);
  m.eok = take(ne);
  m.vw = take(nn);
  m.total = o;
  return m;
}

template <class R>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_tile(Dev d, Geo<R> G, TileDev tp, int s, const double* __restrict__ hs, const uint8_t* __restrict__ dry,
           uint8_t* __restrict__ dry_next, const double* __restrict__ u_in, const double* __restrict__ v_in,
           double* __restrict__ u_out, double* __restrict__ v_out, double* __restrict__ rku_prev,
           double* __restrict__ rkv_prev) {
  extern __shared__ __align__(16) unsigned char tsm[];
  // persistent: each CTA takes tiles blockIdx.x, blockIdx.x + gridDim.x, ...
  for (int t = blockIdx.x; t < tp.ntiles; t += gridDim.x) {
  const int* I = tp.info + (size_t)t * TI_N;
  const int tsid = I[TI_SID];
  if (tsid >= 0 && d.sc[tsid].converged) continue;  // uniform over the CTA
  const int nown = I[TI_NOWN], n1 = I[TI_N1], n2 = I[TI_N2], hoff = I[TI_HOFF], h1off = I[TI_H1OFF];
  const int er0 = I[TI_ER0], nr = I[TI_NR], nb = I[TI_NB], boff = I[TI_BOFF];
  const int noff = I[TI_NOFF], nn = tp.nodes ? I[TI_NN] : 0;
  const int nS = nown + n1 + n2 + (tp.nodes ? I[TI_N3] : 0), nG = nown + n1, nE = nr + nb;
  const int ngm = tp.ng_max, nem = tp.ne_max;
  const int T = d.T, c0 = t * tp.tc;
  const TileSmem L = tile_smem_layout(tp.ns_max, ngm, nem, tp.tc, (int)sizeof(R), tp.nodes ? tp.nn_max : 0);
  double* s_h = reinterpret_cast<double*>(tsm + L.h);
  double* s_z = reinterpret_cast<double*>(tsm + L.z);
  double* s_u = reinterpret_cast<double*>(tsm + L.u);
  double* s_v = reinterpret_cast<double*>(tsm + L.v);
  double* s_fh = reinterpret_cast<double*>(tsm + L.fh);
  double* s_fu = reinterpret_cast<double*>(tsm + L.fu);
  double* s_fv = reinterpret_cast<double*>(tsm + L.fv);
  R* s_dhx = reinterpret_cast<R*>(tsm + L.dhx);
  R* s_dhy = reinterpret_cast<R*>(tsm + L.dhy);
  R* s_f = reinterpret_cast<R*>(tsm + L.f);
  uint8_t* s_dry = tsm + L.dry;
  uint8_t* s_eok = tsm + L.eok;
  double* s_hv = reinterpret_cast<double*>(tsm + L.hv);
  uint8_t* s_vw = tsm + L.vw;

  // A: stage-input state of every local cell
  for (int l = threadIdx.x; l < nS; l += blockDim.x) {
    const int g = l < nown ? c0 + l : tp.halo[hoff + l - nown];
    s_h[l] = hs[g];
    s_z[l] = d.z[g];
    s_u[l] = u_in[g];
    s_v[l] = v_in[g];
    s_dry[l] = dry[g];
  }
  __syncthreads();

  // A2: vertex depths of the tile's nodes from their incident cells (node_depth, the
  // arithmetic of k_node); the tile owning a node's first incident cell writes it out
  if (tp.nodes) {
    for (int ln = threadIdx.x; ln < nn; ln += blockDim.x) {
      const int n = tp.tnode[noff + ln];
      if (!item_live(d, d.node_sid, n)) continue;
      const int b0 = d.n2t_off[n], b1 = d.n2t_off[n + 1];
      const int base = tp.tn_start[noff + ln] - b0;  // tn_cells[base + q] for q in [b0, b1)
      double hv;
      bool wet;
      node_depth(d, n, b0, b1,
                 [&](int q, bool* dk, double* hk, double* zk) {
                   const int k = tp.tn_cells[base + q];
                   *dk = s_dry[k] != 0;
                   *hk = s_h[k];
                   *zk = s_z[k];
                 },
                 &hv, &wet);
      s_hv[ln] = hv;
      s_vw[ln] = wet;
      if (tp.tn_own[noff + ln]) {
        d.hvtx[n] = hv;
        d.vwet[n] = wet;
      }
    }
    __syncthreads();
  }

  // B: gradients and face states of the owned and H1 cells
  const NbShared nbs{s_h, s_z, s_u, s_v, s_dry};
  for (int l = threadIdx.x; l < nG; l += blockDim.x) {
    const bool own = l < nown;
    const int g = own ? c0 + l : tp.halo[hoff + l - nown];
    if (!cell_live(d, g)) continue;
    int t3[3];
    const uint16_t *st, *vt;
    int sst, svt;
    if (own) {
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const uint16_t x = tp.lt3[j * T + g];
        t3[j] = x == kNoLocal ? -1 : (int)x;
      }
      st = tp.lst + g;
      sst = T;
      vt = tp.lvt + g;
      svt = T;
    } else {
      const size_t r = (size_t)(h1off + l - nown);
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const uint16_t x = tp.h1_t3[3 * r + j];
        t3[j] = x == kNoLocal ? -1 : (int)x;
      }
      st = tp.h1_st + (size_t)tp.kst * r;
      sst = 1;
      vt = tp.h1_vt + 3 * r;
      svt = 1;
    }
    R rx[3], ry[3];
    const GradOut<R> gr = cell_gradients<R>(
        d, G, nbs, g, l, t3, [&](int k) { return (int)st[k * sst]; },
        [&](int j) { return tp.nodes ? s_vw[vt[j * svt]] != 0 : d.vwet[d.vert[j * T + g]] != 0; },
        rx, ry);
    if (d.lim != 2) {
#pragma unroll
      for (int j = 0; j < 3; j++) {
        rx[j] = G.rc_x[j * T + g];
        ry[j] = G.rc_y[j * T + g];
      }
    }
    if (own) {
      // the boundary cells' previous-level momentum is zeroed by their k_grad pass
      if (gr.fix && !(d.forder[g] & kOrderHasBc)) {
        rku_prev[g] = kZero;
        rkv_prev[g] = kZero;
      }
      s_dhx[l] = gr.hx;
      s_dhy[l] = gr.hy;
      // the last stage's depth gradient is what the output step's error estimate reads
      // (error_est.f90 etype 2); the boundary cells' comes from their k_grad pass
      if (s == d.K && !(d.forder[g] & kOrderHasBc)) {
        G.delh_x[g] = gr.hx;
        G.delh_y[g] = gr.hy;
      }
    }
    const double h_c = s_h[l];
#pragma unroll
    for (int m = 0; m < 3; m++) {  // edge_state of the three faces (invisc_fluxes.f90:53-81)
      double fh = recon(h_c, gr.hx, rx[m], gr.hy, ry[m]);
      if (fh < kZero) fh = kZero;
      s_fh[m * ngm + l] = fh;
      s_fu[m * ngm + l] = recon(gr.ub, gr.ux, rx[m], gr.uy, ry[m]);
      s_fv[m * ngm + l] = recon(gr.vb, gr.vx, rx[m], gr.vy, ry[m]);
    }
  }
  __syncthreads();

  // C: the flux of every edge of an owned cell
  for (int le = threadIdx.x; le < nE; le += blockDim.x) {
    int e;
    uint32_t lo;
    if (le < nr) {
      e = er0 + le;
      lo = tp.eloc[e];
    } else {
      e = tp.be[boff + le - nr];
      lo = tp.beloc[boff + le - nr];
    }
    bool ok = false;
    if (item_live(d, d.edge_sid, e)) {
      const int a = lo & 0xFFFF, b = lo >> 16;
      const uint8_t sl = d.eslot[e];
      const int ml = sl & 3, mr = (sl >> 2) & 3;
      const bool dl = s_dry[a], dr = s_dry[b];
      const EdgeState fa{s_fh[ml * ngm + a], s_fu[ml * ngm + a], s_fv[ml * ngm + a]};
      const EdgeState fb{s_fh[mr * ngm + b], s_fu[mr * ngm + b], s_fv[mr * ngm + b]};
      R f[3];
      bool bad = false;
      ok = edge_flux<R>(d, dl, dr, fa, fb, s_z[a], s_z[b], s_h[a], s_h[b], G.enx[e], G.eny[e],
                        (dl || dr) ? d.ez0[e] : kZero, f, &bad);
      if (ok) {
        const R len = G.elen[e];
        f[0] = f[0] * len;
        f[1] = f[1] * len;
        f[2] = f[2] * len;
        s_f[le] = f[0];
        s_f[nem + le] = f[1];
        s_f[2 * nem + le] = f[2];
      }
      if ((sl & kEdgeExport) && le < nr) {  // a boundary cell's face: k_flux_bc reads it
        d.eok[e] = ok;
        if (ok) {
          G.efx[e] = f[0];
          G.efx[d.ne + e] = f[1];
          G.efx[2 * d.ne + e] = f[2];
        }
      }
      if (bad) atomicOr(&d.sc[d.edge_sid[e]].status, 2);
    }
    s_eok[le] = ok;
  }
  __syncthreads();

  // D: ordered gather, sources and RK update of the owned cells
  for (int l = threadIdx.x; l < nown; l += blockDim.x) {
    const int c = c0 + l;
    if (!cell_live(d, c)) continue;
    if (d.forder[c] & kOrderHasBc) continue;
    const double h_c = s_h[l];
    const bool dry_c = s_dry[l] != 0;
    const FacesTile<R> fs{tp.lfe, T, c, l, ngm, nem, s_f, s_eok, s_fh, s_fu, s_fv, s_dhx, s_dhy,
                          tp.lwall, tp.nodes ? s_hv : nullptr, d.hvtx, d.wall_p1, d.wall_p2, d.fref,
                          d.forder, d.fkind};
    double p1, p2, p3;
    assemble_phi<R>(d, G, fs, c, h_c, dry_c, &p1, &p2, &p3);
    rk_update(d, s, c, h_c, dry_c, p1, p2, p3, dry_next, u_in, v_in, u_out, v_out);
  }
  __syncthreads();  // the next tile reuses the shared memory
  }
}

#ifndef STORM_FVT_F32_TU
size_t tile_smem_bytes(const TileDev& t, bool mixed) {
  return tile_smem_layout(t.ns_max, t.ng_max, t.ne_max, t.tc, mixed ? 4 : 8, t.nodes ? t.nn_max : 0).total;
}

int tile_blocks_per_sm(bool mixed, size_t smem) {
  int n = 0;
  if (mixed) n = tile_blocks_per_sm_f32(smem);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tile<double>, kTileThreads, smem);
  return n;
}

// The dynamic shared-memory limit is a property of the kernel function (per device),
// shared by every handle: it only ever grows, so a handle that needs less never
// lowers it under another handle's launches.
static int raise_smem_limit(int* per_dev, int bytes) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return bytes;
  if (bytes > per_dev[dev]) per_dev[dev] = bytes;
  return per_dev[dev];
}

void set_tile_smem_limit(int bytes) {
  static int lim[64] = {0};
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  const int b = raise_smem_limit(lim, bytes);
  cudaFuncSetAttribute(k_tile<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  set_tile_smem_attr_f32(b);
}
#endif  // !STORM_FVT_F32_TU

// ---------------------------------------------------------------------------
// After the RK stages: find_dry_cells, fric_terms_impl, hvalve, rk level copy and the
// block partials of the iteration's reductions (solverFVT.f90:335-386, 407-445).
// kHalo: the handle links partitions, and halo cells stay out of the partials.
// u_src/v_src: the velocities of the last stage (the fused path's ping-pong buffer);
// the friction step writes the next iteration's start into d.u_a/d.v_a.
template <bool kHalo>
__global__ void __launch_bounds__(kRedThreads) k_fric(Dev d, const double* __restrict__ u_src,
                                                      const double* __restrict__ v_src) {
  __shared__ double sm[5 * (kRedThreads / 32)];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int T = d.T, K = d.K;
  // one-scenario handles: scenario 0 for the cells below t_real, padding above, with
  // no per-cell scenario id read
  const bool one = d.nscen == 1;
  const int sid = one ? (c < d.t_real ? 0 : -1) : (c < T ? d.cell_sid[c] : -1);
  // a block never spans two scenarios, so this test is uniform over the block
  const int bsid = one ? 0 : d.cell_sid[blockIdx.x * blockDim.x];
  if (d.sc[bsid < 0 ? 0 : bsid].converged) return;
  double st = kZero, sb = kZero, tm = kZero, rm = kZero, dtc = kVlarge;
  if (sid >= 0) {
    const int qk = K * T + c;
    const double h = d.rkh[qk];
    double u = u_src[c], v = v_src[c];
    double ru = d.rku[qk], rv = d.rkv[qk];
    const double h0 = d.rkh[c];  // rkh(i,0), the iteration's starting depth
    double um;
    const bool dry2 = dry_flag(h, u, v, d.h_dry, d.h_wet, &um);
    d.dry_out[c] = dry2;
    const double cd = d.cd[c];
    double rough = kZero;
    switch (d.fric) {
      case 0:
        if (!dry2) rough = kG * cd * cd / pow(h, kOneThird);
        break;
      case 1:
        rough = (cd < kFmachp) ? kVlarge : kG / (cd * cd);
        break;
      case 2:
        rough = cd;
        break;
      case 3:
        if (!dry2) {
          double re = qdiv(um * h, d.visc);
          re = fmax2(re, 1000.0);
          re = fmin2(re, (double)2.5e7f);
          rough = cd;
          if (cd / h > 0.20) rough = 0.20 * h;
          const double ln = log(1.725 / re + pow(rough / (14.8 * h), (double)1.11f));
          rough = 0.204 / (ln * ln);
        }
        break;
      default:
        if (!dry2) {
          rough = pow(100.0 * cd, 0.16666666666666667) / 51.79;
          rough = kG * rough * rough / pow(h, kOneThird);
        }
        break;
    }
    const double dtf = d.steady ? d.sc[sid].delt_fric : d.sc[sid].delt;
    if (!dry2) rough = h / (h + dtf * rough * um);
    u = u * rough;
    v = v * rough;
    if (!dry2) {
      ru = h * u;
      rv = h * v;
    }
    // numerical valve at stage-boundary edges (solverFVT.f90:357-370)
    const uint8_t hm = d.hvalve ? d.hvmask[c] : 0;
    if (hm) {
      bool zero = false;
#pragma unroll
      for (int j = 0; j < 3; j++)
        if (hm & (1u << j)) {
          const int q = j * T + c;
          const double dot = u * d.fnx[q] + v * d.fny[q];
          if (dot < 0) zero = true;
        }
      if (zero) {
        u = kZero;
        v = kZero;
      }
    }
    d.rku[c] = ru;  // rk(:,0) <- rk(:,rkorder) of the next iteration (:138-142)
    d.rkv[c] = rv;
    d.rkh[c] = h;
    d.u_a[c] = u;
    d.v_a[c] = v;
    double um1;
    const bool dry1 = dry_flag(h, u, v, d.h_dry, d.h_wet, &um1);
    d.dry_a[c] = dry1;
    st = (h - h0) * (h - h0);
    sb = h0 * h0;
    tm = h * d.area[c];
    rm = dry2 ? kZero : d.phimax[c];
    const double wc1 = dry1 ? kZero : sqrt(kG * h);
    dtc = d.cfl * d.area[c] / ((um1 + wc1 + SMALL_F) * d.perim[c]);
    if (kHalo && d.halo_mask[c]) {  // a halo copy: its owner counts it
      st = kZero; sb = kZero; tm = kZero; rm = kZero; dtc = kVlarge;
    } else if (!isfinite(h) || !isfinite(u) || !isfinite(v)) {
      atomicOr(&d.sc[sid].status, 1);
    }
  }
  block_reduce5<kRedThreads>(st, sb, tm, rm, dtc, sm, d.part + blockIdx.x, d.nblk_red);
}

#ifndef STORM_FVT_F32_TU
__global__ void __launch_bounds__(kFinalThreads) k_final(Dev d) {
  __shared__ double sm[5 * (kFinalThreads / 32)];
  __shared__ double red[5];
  const int sid = blockIdx.x;
  Scalars* sc = &d.sc[sid];
  if (sc->converged) return;
  double a0 = kZero, a1 = kZero, a2 = kZero, a3 = kZero, a4 = kVlarge;
  const int cnt = sc->blk_cnt;
  // field-major partials ([5][nblk_red]): a warp's loads of one field are coalesced
  const size_t fs = d.nblk_red;
  const double* p0 = d.part + sc->blk_off;
  // rounds of eight partial records in flight per thread (the 2M meander's 7,813
  // records take two); each thread adds its records in increasing order, so the sums
  // round as in a one-at-a-time loop over the same records
  for (int b = threadIdx.x; b < cnt; b += 8 * kFinalThreads) {
    double r[8][5];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int q = b + k * kFinalThreads;
#pragma unroll
      for (int j = 0; j < 5; j++) r[k][j] = q < cnt ? p0[j * fs + q] : kZero;
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      if (b + k * kFinalThreads >= cnt) break;
      a0 = a0 + r[k][0];
      a1 = a1 + r[k][1];
      a2 = a2 + r[k][2];
      a3 = fmax2(a3, r[k][3]);
      a4 = fmin2(a4, r[k][4]);
    }
  }
  block_reduce5<kFinalThreads>(a0, a1, a2, a3, a4, sm, red);
  const double sumtop = red[0], sumbot = red[1], tmass = red[2], rmax_phi = red[3], dtmin = red[4];
  if (threadIdx.x == 0) {
    sc->sumtop = sumtop;
    sc->sumbot = sumbot;
    sc->rmax_phi = rmax_phi;
    sc->iter = sc->iter + 1;
    sc->ttime = sc->ttime + sc->delt;
    double sbot = sumbot;
    if (equals(sbot, kZero)) sbot = kOne;
    sc->rms = sqrt(sumtop / sbot);
    sc->tmass = tmass;
    if (d.steady) {
      sc->rmax = (d.stop_cr == 0) ? rmax_phi : sc->rms;
      sc->stime = (double)sc->iter;
      sc->delt = sc->delt_fric;  // carried into the next iteration's ttime
      if (sc->rmax < d.rstop) sc->converged = 1;
    } else {
      sc->stime = sc->stime + sc->delt;
      sc->rmax = rmax_phi;
      for (int b = 0; b < kMaxBdrDev; b++) {
        sc->qin_it[b] = sc->qin[b];
        sc->hbc_it[b] = sc->hbc[b];
      }
      time_bcs(d, sid, sc->stime);
      sc->delt = (d.dt_op == 0) ? d.cfl : dtmin;
    }
  }
}
#endif  // !STORM_FVT_F32_TU

// ---------------------------------------------------------------------------
// The output pass of solverFVT.f90:389-405 (to_vertices.f90:26-65, ctr2vtx.f90:69-80,
// wetdryvfix.f90, enforce_bcs.f90:37-171, vbc_by_h.f90, error_est.f90 etype 2) after
// an iteration.  The depths come from zeta of the last stage's start (solverFVT.f90:169
// is the only assignment of zeta) and the dry flags of the find_dry_cells call before
// the friction step (:335), as in the reference.

#ifndef STORM_FVT_F32_TU
// to_vertices.f90:26-41: ctr2vtxWSE type 3, cap, positivity_vtx
__global__ void __launch_bounds__(256) k_out_depth(Dev d, OutputArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= d.N) return;
  const double* hs = d.rkh + (size_t)(d.K - 1) * d.T;
  const int b0 = d.n2t_off[n], b1 = d.n2t_off[n + 1];
  const double zv0 = d.zvtx[n];
  double id = kZero, s = kZero, zetaref = zv0;
  int counter = 0;
  for (int q = b0; q < b1; q++) {
    const int k = d.n2t_cell[q];
    if (d.dry_out[k]) continue;
    const double zeta = hs[k] + d.z[k];
    counter++;
    id = id + d.n2t_w[q];
    s = s + d.n2t_w[q] * zeta;
  }
  double zv = counter > 0 ? s / id : zv0;
  for (int q = b0; q < b1; q++) {
    const int k = d.n2t_cell[q];
    if (d.dry_out[k]) continue;
    zetaref = fmax2(hs[k] + d.z[k], zetaref);
  }
  zv = fmin2(zv, zetaref);
  double hv = zv - zv0;
  if (hv < kZero) hv = kZero;
  a.hv[n] = hv;
}
#endif  // !STORM_FVT_F32_TU

// to_vertices.f90:44-55 on the solution (and the next stage's dry flag of a cell whose
// velocity it zeroes), error_est.f90 etype 2
template <class R>
__global__ void __launch_bounds__(256) k_out_cell(Dev d, Geo<R> G, OutputArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.T || d.cell_sid[c] < 0) return;
  const int T = d.T;
  const int n1 = d.vert[c], n2 = d.vert[(size_t)T + c], n3 = d.vert[2 * (size_t)T + c];
  const double h = d.rkh[c];
  if (!d.dry_out[c]) {
    const bool flag = (a.hv[n1] > d.h_dry) && (a.hv[n2] > d.h_dry) && (a.hv[n3] > d.h_dry);
    if (!flag) {
      d.u_a[c] = kZero;
      d.v_a[c] = kZero;
      double um;
      d.dry_a[c] = dry_flag(h, kZero, kZero, d.h_dry, d.h_wet, &um);
    }
  }
  if (a.e_est) {
    double e = kZero;
    if (!(h < d.h_dry)) {
      const double x1 = d.node_x[n1], x2 = d.node_x[n2], x3 = d.node_x[n3];
      const double y1 = d.node_y[n1], y2 = d.node_y[n2], y3 = d.node_y[n3];
      const double z1 = d.zvtx[n1], z2 = d.zvtx[n2], z3 = d.zvtx[n3];
      const double gzx = (z1 * (y2 - y3) + z2 * (y3 - y1) + z3 * (y1 - y2)) * kHalf / d.area[c];
      const double gzy = (z1 * (x3 - x2) + z2 * (x1 - x3) + z3 * (x2 - x1)) * kHalf / d.area[c];
      const double l = d.perim[c] * kOneThird;
      const double gx = gzx + (double)G.delh_x[c], gy = gzy + (double)G.delh_y[c];
      e = sqrt(gx * gx + gy * gy) * l / (d.z[c] + h);
    }
    a.e_est[c] = e;
  }
}

#ifndef STORM_FVT_F32_TU
// ctr2vtx type 3 of u, v and cd with the normalised weights (c2v_setup.f90:113-117),
// wetdryvfix (btype 0), the dry-vertex zeroing of to_vertices.f90:58-61
__global__ void __launch_bounds__(256) k_out_vel(Dev d, OutputArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= d.N) return;
  const int b0 = d.n2t_off[n], b1 = d.n2t_off[n + 1];
  double tdist = kZero;
  for (int q = b0; q < b1; q++) tdist = tdist + d.n2t_w[q];
  double su = kZero, sv = kZero, scd = kZero;
  bool wett = false, dryt = false;
  for (int q = b0; q < b1; q++) {
    const int k = d.n2t_cell[q];
    const double w = d.n2t_w[q] / tdist;
    su = su + w * d.u_a[k];
    sv = sv + w * d.v_a[k];
    scd = scd + w * d.cd[k];
    if (d.dry_out[k]) dryt = true;
    else wett = true;
  }
  if (d.btype == 0 && wett && dryt) {
    su = kZero;
    sv = kZero;
  }
  if (a.hv[n] < d.h_dry) {
    su = kZero;
    sv = kZero;
  }
  a.uv[n] = su;
  a.vv[n] = sv;
  if (a.cdv) a.cdv[n] = scd;
}

// enforce_bcs.f90:37-94, the outflow strings in order (one thread: the strings may
// share end nodes)
__global__ void k_out_outflow(Dev d, OutputArgs a) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int b = 0; b < a.n_out; b++) {
    const int ty = a.out_type[b];
    if (ty == 1)  // :44-56: the relaxed update is overwritten by the instantaneous one
      for (int i = a.out_off[b]; i < a.out_off[b + 1]; i++) {
        const int j = a.out_node[i];
        a.hv[j] = fmax2(kZero, a.hbc[b] - d.zvtx[j]);
      }
    if (!((ty == 1 && d.hvalve) || ty == 0)) continue;
    for (int i = a.out_off[b]; i < a.out_off[b + 1]; i++) {
      const int j = a.out_node[i];
      const double dot = a.uv[j] * a.hn[2 * i] + a.vv[j] * a.hn[2 * i + 1];
      if (dot < kZero) {
        a.uv[j] = kZero;
        a.vv[j] = kZero;
      }
    }
  }
}

// enforce_bcs.f90:97-121, walls then dry nodes
__global__ void __launch_bounds__(256) k_out_walls(Dev d, OutputArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_wall) return;
  const int p = a.wall_node[i];
  if (d.btype == 0) {
    a.uv[p] = kZero;
    a.vv[p] = kZero;
  } else {
    const double tx = a.wtang[2 * i], ty = a.wtang[2 * i + 1];
    const double dot = a.uv[p] * tx + a.vv[p] * ty;
    a.uv[p] = dot * tx;
    a.vv[p] = dot * ty;
  }
}
__global__ void __launch_bounds__(256) k_out_drynodes(Dev d, OutputArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= d.N) return;
  if (a.hv[n] < d.h_dry) {
    a.uv[n] = kZero;
    a.vv[n] = kZero;
  }
}
#endif  // !STORM_FVT_F32_TU

// enforce_bcs.f90:124-169 with vbc_by_h.f90 for one inflow string, serial in node order
// as the reference (the sums of vbc_by_h keep their order)
static __device__ void out_inflow_string(const Dev& d, const OutputArgs& a, int b) {
  const int o = a.in_off[b], n = a.in_off[b + 1] - o;
  const int vt = a.in_type[b];
  const double qin = a.qin[b];
  if (vt == 0 || vt == 3) {
    for (int i = 0; i < n; i++) {
      const int p = a.in_node[o + i];
      if (a.hv[p] > d.h_dry) {
        a.uv[p] = vt == 0 ? qin * a.pn[2 * (o + i)] : qin;
        a.vv[p] = vt == 0 ? qin * a.pn[2 * (o + i) + 1] : (a.qin2 ? a.qin2[b] : kZero);
      }
    }
    return;
  }
  if (vt != 1 && vt != 5) return;
  // vbc_by_h: v_inflow(i), two passes over the string, all sums in node order
  double ht = kZero, at = kZero;
  for (int i = 0; i + 1 < n; i++) {
    const double h1 = a.hv[a.in_node[o + i]], h2 = a.hv[a.in_node[o + i + 1]];
    const double ai = a.lin[o + i] * (h1 + h2) * kHalf;
    ht = ht + (h1 + h2) * kHalf;
    at = at + ai;
  }
  // u_inflow(i) = half*(h(i)+h(i+1))*qin/ht/at; v(i) = half*(u(i-1)+u(i)) for wet inner nodes
  auto hin = [&](int i) { return a.hv[a.in_node[o + i]]; };
  auto u1 = [&](int i) { return kHalf * (hin(i) + hin(i + 1)) * qin / ht / at; };
  auto v1 = [&](int i) { return (i >= 1 && i <= n - 2 && hin(i) > d.h_dry) ? kHalf * (u1(i - 1) + u1(i)) : kZero; };
  double q = kZero;
  for (int i = 0; i + 1 < n; i++) {
    const double ui = kHalf * (v1(i) + v1(i + 1));
    q = q + ui * (a.lin[o + i] * (hin(i) + hin(i + 1)) * kHalf);
  }
  auto v2 = [&](int i) { return (i >= 1 && i <= n - 2 && hin(i) > d.h_dry) ? v1(i) * qin / q : v1(i); };
  for (int i = 0; i < n; i++) {
    const int p = a.in_node[o + i];
    if (a.hv[p] > d.h_dry) {
      const double vi = v2(i);
      a.uv[p] = vi * a.pn[2 * (o + i)];
      a.vv[p] = vi * a.pn[2 * (o + i) + 1];
    }
  }
}
#ifndef STORM_FVT_F32_TU
__global__ void k_out_inflow(Dev d, OutputArgs a) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int b = 0; b < a.n_in; b++) out_inflow_string(d, a, b);
}

// The next iteration's CFL dt after the output pass zeroed velocities: the reference
// computes it at the start of that iteration from the current u, v (deltatFVT), so
// the partials of k_fric are recomputed (same expression) and reduced again.
__global__ void __launch_bounds__(kRedThreads) k_out_dt(Dev d) {
  __shared__ double sm[kRedThreads / 32];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double dtc = kVlarge;
  if (c < d.T && d.cell_sid[c] >= 0) {
    const double h = d.rkh[c];
    double um1;
    const bool dry1 = dry_flag(h, d.u_a[c], d.v_a[c], d.h_dry, d.h_wet, &um1);
    const double wc1 = dry1 ? kZero : sqrt(kG * h);
    dtc = d.cfl * d.area[c] / ((um1 + wc1 + SMALL_F) * d.perim[c]);
  }
  const double r = block_min<kRedThreads>(dtc, sm);
  if (threadIdx.x == 0) d.part[4 * (size_t)d.nblk_red + blockIdx.x] = r;
}
__global__ void __launch_bounds__(kRedThreads) k_out_dtfinal(Dev d) {
  __shared__ double sm[kRedThreads / 32];
  Scalars* sc = &d.sc[blockIdx.x];
  double a4 = kVlarge;
  for (int b = threadIdx.x; b < sc->blk_cnt; b += blockDim.x) a4 = fmin2(a4, d.part[4 * (size_t)d.nblk_red + sc->blk_off + b]);
  const double dtmin = block_min<kRedThreads>(a4, sm);
  if (threadIdx.x == 0) sc->delt = dtmin;
}

void launch_output(const Dev& d, const Geo<double>& Gd, const Geo<float>& Gf, bool mixed, const OutputArgs& a,
                   cudaStream_t st) {
  const int gN = (d.N + 255) / 256, gT = (d.T + 255) / 256;
  k_out_depth<<<gN, 256, 0, st>>>(d, a);
  if (mixed) launch_out_cell_f32(d, Gf, a, gT, st);
  else k_out_cell<double><<<gT, 256, 0, st>>>(d, Gd, a);
  k_out_vel<<<gN, 256, 0, st>>>(d, a);
  if (a.n_out > 0) k_out_outflow<<<1, 32, 0, st>>>(d, a);
  if (a.n_wall > 0) k_out_walls<<<(a.n_wall + 255) / 256, 256, 0, st>>>(d, a);
  k_out_drynodes<<<gN, 256, 0, st>>>(d, a);
  if (a.n_in > 0) k_out_inflow<<<1, 32, 0, st>>>(d, a);
  if (!d.steady && d.dt_op == 1) {
    k_out_dt<<<d.nblk_red, kRedThreads, 0, st>>>(d);
    k_out_dtfinal<<<d.nscen, kRedThreads, 0, st>>>(d);
  }
}
#endif  // !STORM_FVT_F32_TU

// Discharge of every culvert (cvdisch.f90:19-49), one thread per culvert, after the
// stage's gradients: the headwater at the inlet is the stage reconstructed from the
// inlet cell's centroid (zeta + (delh + delz) . rcv) minus the invert elevation, and
// the discharge is interpolated linearly in the culvert's performance curve.
template <class R>
__global__ void k_culvert(Dev d, Geo<R> G, const double* __restrict__ hs, const uint8_t* __restrict__ dry) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.ncv) return;
  double src = kZero;
  const int c = d.cv_in[i];
  if (!dry[c]) {
    const double zeta = hs[c] + d.z[c];
    const double dhx = (double)G.delh_x[c], dhy = (double)G.delh_y[c];
    double head = zeta + (dhx + d.delz_x[c]) * d.cv_rx[i] + (dhy + d.delz_y[c]) * d.cv_ry[i];
    head = head - d.cv_zinv[i];
    if (!(head < d.h_dry)) {
      const double* hd = d.cv_head + (size_t)i * d.cv_ld;
      const double* q = d.cv_q + (size_t)i * d.cv_ld;
      const int nt = d.cv_n[i];
      if (head < hd[0]) {
        src = q[0];
      } else if (head >= hd[nt - 1]) {
        src = q[nt - 1];
      } else {
        for (int j = 1; j <= nt - 1; j++)
          if (head < hd[j]) {
            const double t = (head - hd[j - 1]) / (hd[j] - hd[j - 1]);
            src = q[j] * t + q[j - 1] * (kOne - t);
            break;
          }
      }
    }
  }
  d.cvsrc[i] = src;
}

// ---------------------------------------------------------------------------
// Linked partitions of one mesh (storm_fvt_link_partitions).  The scenarios share
// one clock, so the first one's stop flag stands for all.

#ifndef STORM_FVT_F32_TU
// Every halo cell takes its owner's values of one RK level, the velocities and up to
// two flag arrays.
__global__ void __launch_bounds__(256) k_halo(Dev d, int level, uint8_t* f1, uint8_t* f2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.nhalo || d.sc[0].converged) return;
  const int dst = d.halo_dst[i], src = d.halo_src[i];
  const size_t off = (size_t)level * d.T;
  d.rkh[off + dst] = d.rkh[off + src];
  d.rku[off + dst] = d.rku[off + src];
  d.rkv[off + dst] = d.rkv[off + src];
  d.u_a[dst] = d.u_a[src];
  d.v_a[dst] = d.v_a[src];
  if (f1) f1[dst] = f1[src];
  if (f2) f2[dst] = f2[src];
}

// Unsteady runs: the first dt after a state is set comes from each part's own CFL
// minimum; every iteration starts from the smallest (later ones are already equal).
__global__ void k_link_dt(Dev d) {
  if (threadIdx.x != 0 || d.sc[0].converged) return;
  double dmin = kVlarge;
  for (int s = 0; s < d.nscen; s++) dmin = fmin2(dmin, d.sc[s].delt);
  for (int s = 0; s < d.nscen; s++) d.sc[s].delt = dmin;
}

// Steady runs: the friction step of every part uses the local dt of element n_elems
// of the whole mesh (solverFVT.f90:155 and :335-356), set in the part that owns it.
__global__ void k_link_fric(Dev d) {
  if (threadIdx.x != 0 || d.sc[0].converged) return;
  const double v = d.sc[d.fric_scen].delt_fric;
  for (int s = 0; s < d.nscen; s++) d.sc[s].delt_fric = v;
}

// After k_final: the residual, mass and dt of the whole mesh from the parts' sums
// (added in scenario order), and one stop test for all parts.
__global__ void k_link(Dev d) {
  if (threadIdx.x != 0 || d.sc[0].converged) return;
  double top = kZero, bot = kZero, tm = kZero, rmx = kZero, dmin = kVlarge;
  for (int s = 0; s < d.nscen; s++) {
    top = top + d.sc[s].sumtop;
    bot = bot + d.sc[s].sumbot;
    tm = tm + d.sc[s].tmass;
    rmx = fmax2(rmx, d.sc[s].rmax_phi);
    dmin = fmin2(dmin, d.sc[s].delt);
  }
  double sbot = bot;
  if (equals(sbot, kZero)) sbot = kOne;
  const double rms = sqrt(top / sbot);
  const double rmax = (d.steady && d.stop_cr != 0) ? rms : rmx;
  const int conv = d.steady && rmax < d.rstop;
  for (int s = 0; s < d.nscen; s++) {
    Scalars* sc = &d.sc[s];
    sc->rms = rms;
    sc->tmass = tm;
    sc->rmax = rmax;
    sc->converged = conv;
    if (!d.steady && d.dt_op != 0) sc->delt = dmin;
  }
}
#endif  // !STORM_FVT_F32_TU

// ---------------------------------------------------------------------------
// One part of a mesh per process (storm_fvt_iter_*): the caller moves the halo values
// between the processes and reduces dt and the sums; these kernels set the agreed
// scalars and pack / unpack the exchanged cells.

#ifndef STORM_FVT_F32_TU
// which 0: the iteration's dt; 1: the steady friction dt (element n_elems of the mesh)
__global__ void k_part_scalar(Dev d, int which, double v) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (which == 0) d.sc[0].delt = v;
  else d.sc[0].delt_fric = v;
}

// out[6][n]: h (= rkh of the level), u, v, rkh, rku, rkv of the listed slots
__global__ void __launch_bounds__(256) k_pack(Dev d, int level, int n, const int32_t* __restrict__ slots,
                                              const double* __restrict__ u, const double* __restrict__ v,
                                              double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = slots[k];
  const size_t q = (size_t)level * d.T + c;
  out[k] = d.rkh[q];
  out[n + k] = u[c];
  out[2 * (size_t)n + k] = v[c];
  out[3 * (size_t)n + k] = d.rkh[q];
  out[4 * (size_t)n + k] = d.rku[q];
  out[5 * (size_t)n + k] = d.rkv[q];
}

// The received values into the listed (halo) slots, and their dry flags as the owner
// derived them from the same state (find_dry_cells, as rk_update and k_fric do)
__global__ void __launch_bounds__(256) k_unpack(Dev d, int level, int n, const int32_t* __restrict__ slots,
                                                const double* __restrict__ in, double* __restrict__ u,
                                                double* __restrict__ v, uint8_t* __restrict__ dry) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = slots[k];
  const size_t q = (size_t)level * d.T + c;
  const double hh = in[3 * (size_t)n + k], uu = in[n + k], vv = in[2 * (size_t)n + k];
  d.rkh[q] = hh;
  d.rku[q] = in[4 * (size_t)n + k];
  d.rkv[q] = in[5 * (size_t)n + k];
  u[c] = uu;
  v[c] = vv;
  double um;
  dry[c] = dry_flag(hh, uu, vv, d.h_dry, d.h_wet, &um);
}

// The iteration's residual, mass, max |phi| and stop test from the sums of all parts
// (k_final's expressions with the whole mesh's sums).
__global__ void k_part_finish(Dev d, double top, double bot, double tm, double rmx) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  Scalars* sc = &d.sc[0];
  double sbot = bot;
  if (equals(sbot, kZero)) sbot = kOne;
  sc->rms = sqrt(top / sbot);
  sc->tmass = tm;
  sc->sumtop = top;
  sc->sumbot = bot;
  sc->rmax_phi = rmx;
  if (d.steady) {
    sc->rmax = (d.stop_cr == 0) ? rmx : sc->rms;
    sc->converged = sc->rmax < d.rstop;
  } else {
    sc->rmax = rmx;
  }
}

void launch_part_scalar(const Dev& d, int which, double v, cudaStream_t st) {
  k_part_scalar<<<1, 32, 0, st>>>(d, which, v);
}
void launch_pack(const Dev& d, int level, int n, const int32_t* slots, const double* u, const double* v,
                 double* out, cudaStream_t st) {
  if (n > 0) k_pack<<<(n + 255) / 256, 256, 0, st>>>(d, level, n, slots, u, v, out);
}
void launch_unpack(const Dev& d, int level, int n, const int32_t* slots, const double* in, double* u, double* v,
                   uint8_t* dry, cudaStream_t st) {
  if (n > 0) k_unpack<<<(n + 255) / 256, 256, 0, st>>>(d, level, n, slots, in, u, v, dry);
}
void launch_part_finish(const Dev& d, const double* sums, cudaStream_t st) {
  k_part_finish<<<1, 32, 0, st>>>(d, sums[0], sums[1], sums[2], sums[3]);
}

void launch_halo(const Dev& d, int level, uint8_t* f1, uint8_t* f2, cudaStream_t st) {
  k_halo<<<(d.nhalo + 255) / 256, 256, 0, st>>>(d, level, f1, f2);
}
void launch_link_fric(const Dev& d, cudaStream_t st) { k_link_fric<<<1, 32, 0, st>>>(d); }
void launch_fric(const Dev& d, const double* u_src, const double* v_src, cudaStream_t st) {
  if (d.nhalo > 0) k_fric<true><<<d.nblk_red, kRedThreads, 0, st>>>(d, u_src, v_src);
  else k_fric<false><<<d.nblk_red, kRedThreads, 0, st>>>(d, u_src, v_src);
}
void launch_link_dt(const Dev& d, cudaStream_t st) { k_link_dt<<<1, 32, 0, st>>>(d); }
void launch_link(const Dev& d, cudaStream_t st) { k_link<<<1, 32, 0, st>>>(d); }
#endif  // !STORM_FVT_F32_TU

// ---------------------------------------------------------------------------
// Host launchers of the templated stage kernels (api.cu is not templated).
template <class R>
static void launch_stage_t(const StageLaunch& L, const Dev& d, const Geo<R>& G) {
  switch (L.which) {
    case STAGE_GRAD:
      k_grad<R, false><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry, L.rku_prev, L.rkv_prev, L.u_in, L.v_in);
      break;
    case STAGE_GRAD_BC:
      k_grad<R, true><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry, L.rku_prev, L.rkv_prev, L.u_in, L.v_in);
      break;
    case STAGE_BC:
      k_bc<R><<<L.grid, L.block, L.smem, L.stream>>>(d, G, L.hs, L.dry, L.u_in, L.v_in);
      break;
    case STAGE_EFLUX:
      k_eflux<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry, L.u_in, L.v_in);
      break;
    case STAGE_FLUX:
      k_flux<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.s, L.hs, L.dry, L.dry_next, L.u_in, L.v_in, L.u_out,
                                                   L.v_out);
      break;
    case STAGE_FLUX_BC:
      k_flux_bc<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.s, L.hs, L.dry, L.dry_next, L.u_in, L.v_in, L.u_out,
                                                      L.v_out);
      break;
    case STAGE_PHI:
      k_flux_phi<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry, L.u_in, L.v_in, 0);
      break;
    case STAGE_PHI_BC:
      k_flux_phi<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry, L.u_in, L.v_in, 1);
      break;
    case STAGE_CULVERT:
      k_culvert<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry);
      break;
    case STAGE_TILE:
      k_tile<R><<<L.grid, L.block, L.smem, L.stream>>>(d, G, *L.tiles, L.s, L.hs, L.dry, L.dry_next, L.u_in, L.v_in,
                                                        L.u_out, L.v_out, L.rku_prev, L.rkv_prev);
      break;
  }
}

#ifndef STORM_FVT_F32_TU
void launch_stage(const StageLaunch& L, const Dev& d, const Geo<double>& Gd, const Geo<float>& Gf, bool mixed) {
  if (L.which == STAGE_UPDATE) {  // not templated: the same kernel on both paths
    k_update<<<L.grid, L.block, 0, L.stream>>>(d, L.s, L.hs, L.dry, L.dry_next);
    return;
  }
  if (mixed) launch_stage_f32(L, d, Gf);
  else launch_stage_t<double>(L, d, Gd);
}

void launch_node(const Dev& d, const double* hs, const uint8_t* dry, const int32_t* list, int n, int block,
                 cudaStream_t st) {
  const int cnt = list ? n : d.N;
  if (cnt > 0) k_node<<<(cnt + block - 1) / block, block, 0, st>>>(d, hs, dry, list, n);
}

void launch_rsavg(const Dev& d, int off, int cnt, cudaStream_t st) {
  if (cnt > 0) k_rsavg<<<(cnt + 255) / 256, 256, 0, st>>>(d, off, cnt);
}

void set_bc_smem_limit(int bytes) {
  static int lim[64] = {0};
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  const int b = raise_smem_limit(lim, bytes);
  cudaFuncSetAttribute(k_bc<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  set_bc_smem_attr_f32(b);
}
#endif  // !STORM_FVT_F32_TU

#ifdef STORM_FVT_F32_TU
int tile_blocks_per_sm_f32(size_t smem) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tile<float>, kTileThreads, smem);
  return n;
}
void set_tile_smem_attr_f32(int bytes) {
  cudaFuncSetAttribute(k_tile<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
void set_bc_smem_attr_f32(int bytes) {
  cudaFuncSetAttribute(k_bc<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
void launch_stage_f32(const StageLaunch& L, const Dev& d, const Geo<float>& G) { launch_stage_t<float>(L, d, G); }
void launch_out_cell_f32(const Dev& d, const Geo<float>& G, const OutputArgs& a, int grid, cudaStream_t st) {
  k_out_cell<float><<<grid, 256, 0, st>>>(d, G, a);
}
#endif  // STORM_FVT_F32_TU

}  // namespace storm
