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
__device__ __forceinline__ float qdiv(float a, float b) {
  float r;
  if (a == 0.0f && b != 0.0f && b == b)
    r = __int_as_float((__float_as_int(a) ^ __float_as_int(b)) & (int)0x80000000u);
  else
    r = a / b;
  return r;
}

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

constexpr int kRedThreads = 256;

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
  if (threadIdx.x == 0) d.part[8 * (c0 / kRedThreads + blockIdx.x) + 4] = r;
}

// One block per listed scenario: initial scalars and the first dt.
__global__ void __launch_bounds__(kRedThreads) k_init_final(Dev d, int sid) {
  __shared__ double sm[kRedThreads / 32];
  Scalars* sc = &d.sc[sid];
  double m = kVlarge;
  for (int b = threadIdx.x; b < sc->blk_cnt; b += blockDim.x) m = fmin2(m, d.part[8 * (sc->blk_off + b) + 4]);
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

// ---------------------------------------------------------------------------
// Vertex water surface and depth of one stage.
__global__ void __launch_bounds__(256) k_node(Dev d, const double* __restrict__ hs, const uint8_t* __restrict__ dry) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= d.N) return;
  const int sid = d.node_sid[n];
  if (d.sc[sid].converged) return;
  const int b0 = d.n2t_off[n], b1 = d.n2t_off[n + 1];
  const double zv0 = d.zvtx[n];
  double id = kZero, a = kZero, zetaref = zv0;
  int counter = 0;
  for (int q = b0; q < b1; q++) {
    const int k = d.n2t_cell[q];
    if (dry[k]) continue;
    const double zeta = hs[k] + d.z[k];
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
  d.vwet[n] = hv > d.h_dry;
  const int b = d.node_hbc[n];
  if (b >= 0) hv = fmax2(kZero, d.sc[sid].hbc[b] - zv0);
  d.hvtx[n] = hv;
}

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

template <class R>
__global__ void __launch_bounds__(256, 5) k_grad(Dev d, Geo<R> G, const double* __restrict__ hs,
                                              const uint8_t* __restrict__ dry, double* __restrict__ rku_prev,
                                              double* __restrict__ rkv_prev) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.T) return;
  const int sid = d.cell_sid[c];
  if (sid < 0 || d.sc[sid].converged) return;
  const int T = d.T;
  const double zeta_c = hs[c] + d.z[c];
  const double u_c = d.u_a[c], v_c = d.v_a[c];
  // face neighbours and vertices first: their loads (and the flags read through them
  // below) are in flight while the stencil is gathered
  int t3[3], vt[3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    t3[j] = d.t2t3[(size_t)j * T + c];
    vt[j] = d.vert[(size_t)j * T + c];
  }
  const bool dry_c = dry[c];
  R hx = R(0), hy = R(0), ux = R(0), uy = R(0), vx = R(0), vy = R(0);
  if (d.lim == 1 || d.lim == 2) {
    R dz = R(0), ez = R(0), du = R(0), eu = R(0), dv = R(0), ev = R(0);
    const int n = d.nst[c];
    int k0 = 0;
    if (n >= 3) {  // interior cells: the three face neighbours, all gathers issued together
      int jj[3];
      R w[3], dx[3], dy[3], pz[3], pu[3], pv[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const size_t q = (size_t)k * T + c;
        jj[k] = d.st_id[q];
        w[k] = G.st_w[q];
        dx[k] = G.st_dx[q];
        dy[k] = G.st_dy[q];
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        pz[k] = (R)((hs[jj[k]] + d.z[jj[k]]) - zeta_c);
        pu[k] = (R)(d.u_a[jj[k]] - u_c);
        pv[k] = (R)(d.v_a[jj[k]] - v_c);
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        dz = dz + w[k] * pz[k] * dx[k];
        ez = ez + w[k] * pz[k] * dy[k];
        du = du + w[k] * pu[k] * dx[k];
        eu = eu + w[k] * pu[k] * dy[k];
        dv = dv + w[k] * pv[k] * dx[k];
        ev = ev + w[k] * pv[k] * dy[k];
      }
      k0 = 3;
    }
    for (int k = k0; k < n; k++) {
      const size_t q = (size_t)k * T + c;
      const int j = d.st_id[q];
      const R w = G.st_w[q], dx = G.st_dx[q], dy = G.st_dy[q];
      const R pz = (R)((hs[j] + d.z[j]) - zeta_c);
      const R pu = (R)(d.u_a[j] - u_c);
      const R pv = (R)(d.v_a[j] - v_c);
      dz = dz + w * pz * dx;
      ez = ez + w * pz * dy;
      du = du + w * pu * dx;
      eu = eu + w * pu * dy;
      dv = dv + w * pv * dx;
      ev = ev + w * pv * dy;
    }
    const R ai = G.lsq_a[c], bi = G.lsq_b[c], ci = G.lsq_c[c], det = G.lsq_det[c];
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
      const size_t q = (size_t)j * T + c;
      const int k = t3[j];
      const R rx = G.rc_x[q], ry = G.rc_y[q];
      const double qz = k < 0 ? zeta_c : hs[k] + d.z[k];
      const double qu = k < 0 ? u_c : d.u_a[k];
      const double qv = k < 0 ? v_c : d.v_a[k];
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
  if (!dry_c) {
    // hgradfix2.f90:48-98
    bool setgrad = zeta_c < d.zmax[c];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const int l = t3[j];
      if (l < 0) continue;
      if (dry[l] && d.z[l] < zeta_c) setgrad = false;
    }
    if (setgrad) {
      hx = -G.delz_x[c];
      hy = -G.delz_y[c];
      ub = kZero;
      vb = kZero;
      rku_prev[c] = kZero;
      rkv_prev[c] = kZero;
      ux = R(0); uy = R(0); vx = R(0); vy = R(0);
    }
    // to_vertices.f90:44-55
    bool flag = true;
#pragma unroll
    for (int j = 0; j < 3; j++) flag = flag && d.vwet[vt[j]];
    if (!flag) {
      ub = kZero;
      vb = kZero;
    }
  }
  G.delh_x[c] = hx; G.delh_y[c] = hy;
  G.delu_x[c] = ux; G.delu_y[c] = uy;
  G.delv_x[c] = vx; G.delv_y[c] = vy;
  d.u_b[c] = ub;
  d.v_b[c] = vb;
}

// ---------------------------------------------------------------------------
// Open-boundary fluxes (invisc_fluxes.f90:218-238), one CTA per boundary.  The
// per-edge arithmetic runs on all threads; the sums the reference accumulates
// serially (atotal, newatotal, qtotal, cqin3/cqout3) are added by thread 0 in
// string order, so they round exactly as the reference's loops.
constexpr int kBcThreads = 128;

template <class R>
__global__ void __launch_bounds__(kBcThreads) k_bc(Dev d, Geo<R> G, const double* __restrict__ hs,
                                                   const uint8_t* __restrict__ dry) {
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
    const size_t q = (size_t)m * T + i;
    d.bc_rec[off + e] = recon(hs[i], G.delh_x[i], G.rc_x[q], G.delh_y[i], G.rc_y[q]);
    d.bc_rec[NB + off + e] = recon(d.u_b[i], G.delu_x[i], G.rc_x[q], G.delu_y[i], G.rc_y[q]);
    d.bc_rec[2 * NB + off + e] = recon(d.v_b[i], G.delv_x[i], G.rc_x[q], G.delv_y[i], G.rc_y[q]);
  }
  __syncthreads();
  auto put = [&](int e, double c1, double c2, double c3) {
    d.bc_c[off + e] = c1;
    d.bc_c[NB + off + e] = c2;
    d.bc_c[2 * NB + off + e] = c3;
  };
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
__device__ __forceinline__ EdgeState edge_state(const Dev& d, const Geo<R>& G, const double* __restrict__ hs, int x,
                                                int m) {
  const size_t q = (size_t)m * d.T + x;
  const R rx = G.rc_x[q], ry = G.rc_y[q];
  EdgeState s;
  s.h = recon(hs[x], G.delh_x[x], rx, G.delh_y[x], ry);
  if (s.h < kZero) s.h = kZero;
  s.u = recon(d.u_b[x], G.delu_x[x], rx, G.delu_y[x], ry);
  s.v = recon(d.v_b[x], G.delv_x[x], rx, G.delv_y[x], ry);
  return s;
}

// invisc_fluxes.f90:39-147 for the interior edge between L=e(1) (slot ml) and
// R=e(2) (slot mr); returns false when the edge is skipped.  The wet/dry tests and
// the I1 stage comparison run on the FP64 face states; the flux function in R.
template <class R>
__device__ __forceinline__ bool interior_flux(const Dev& d, const Geo<R>& G, const double* __restrict__ hs,
                                              const uint8_t* __restrict__ dry, int L, int ml, int Rc, int mr, R nx,
                                              R ny, double z0e, R* f, bool* bad) {
  const bool dl = dry[L], dr = dry[Rc];
  if (dl && dr) return false;
  double hleft = kZero, uleft = kZero, vleft = kZero, hright = kZero, uright = kZero, vright = kZero;
  if (!dl) {
    EdgeState s = edge_state(d, G, hs, L, ml);
    hleft = s.h; uleft = s.u; vleft = s.v;
  }
  if (!dr) {
    EdgeState s = edge_state(d, G, hs, Rc, mr);
    hright = s.h; uright = s.u; vright = s.v;
  }
  if (hleft < d.h_dry && hright < d.h_dry) return false;
  bool set_wall = false;
  if (dl || dr) {  // ALGORITHM I1
    double h0 = fmax2(hright, hleft);
    h0 = h0 + z0e;
    if (dl)
      if (d.z[L] + d.h_wet > h0) { set_wall = true; hleft = hright; }
    if (dr)
      if (d.z[Rc] + d.h_wet > h0) { set_wall = true; hright = hleft; }
  }
  if (set_wall) {
    f[0] = R(kZero);
    const R hw = (R)fmax2(hleft, hright);
    f[1] = R(kHalf) * R(kG) * hw * hw * nx;
    f[2] = R(kHalf) * R(kG) * hw * hw * ny;
  } else if (d.flux == STORM_FLUX_HLL) {
    flux_hll<R>(nx, ny, (R)hleft, (R)uleft, (R)vleft, (R)hright, (R)uright, (R)vright, (R)d.h_dry, f, bad);
  } else if (d.flux == STORM_FLUX_RUSANOV) {
    const R cl = dl ? R(kZero) : (R)sqrt(kG * hs[L]);  // wavec (solverFVT.f90:180-181)
    const R cr = dr ? R(kZero) : (R)sqrt(kG * hs[Rc]);
    flux_rusanov<R>(nx, ny, (R)hleft, (R)uleft, (R)vleft, cl, (R)hright, (R)uright, (R)vright, cr, f);
  } else {
    flux_roe<R>(nx, ny, (R)hleft, (R)uleft, (R)vleft, (R)hright, (R)uright, (R)vright, f);
  }
  return true;
}

// Interior-edge fluxes of one stage (invisc_fluxes.f90:39-147), one thread per edge:
// the flux of edge k is evaluated once, in the reference's orientation (left =
// edges(k)%e(1)), and stored as f*length, the amount the reference subtracts from
// phi(e(1),:) and adds to phi(e(2),:).
template <class R>
__global__ void __launch_bounds__(128, 8) k_eflux(Dev d, Geo<R> G, const double* __restrict__ hs,
                                               const uint8_t* __restrict__ dry) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.ne) return;
  const int sid = d.edge_sid[e];
  if (d.sc[sid].converged) return;
  const int L = d.eL[e], Rc = d.eR[e];
  const uint8_t sl = d.eslot[e];
  R f[3];
  bool bad = false;
  const bool ok = interior_flux<R>(d, G, hs, dry, L, sl & 3, Rc, (sl >> 2) & 3, G.enx[e], G.eny[e],
                                   (dry[L] || dry[Rc]) ? d.ez0[e] : kZero, f, &bad);
  d.eok[e] = ok;
  if (ok) {
    const R len = G.elen[e];
    G.efx[e] = f[0] * len;
    G.efx[d.ne + e] = f[1] * len;
    G.efx[2 * d.ne + e] = f[2] * len;
  }
  if (bad) atomicOr(&d.sc[sid].status, 2);
}

// bed_slope_STD.f90:23-70 with adjustZb.f90:41-70: the amounts g*h*gradzb*area that
// are subtracted from phi(i,2:3).  The adjust test (a negative reconstructed vertex
// depth) and the adjusted gradient run in double on both paths.
__device__ __forceinline__ void bed_source(const Dev& d, const Geo<double>& G, int c, double h_c, double* s2,
                                           double* s3) {
  const int T = d.T;
  const double dhx = G.delh_x[c], dhy = G.delh_y[c], xc = d.xc[c], yc = d.yc[c];
  int vid[3];
  double hp[3];
  bool adjust = false;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    vid[i] = d.vert[(size_t)i * T + c];
    hp[i] = h_c + dhx * (d.node_x[vid[i]] - xc) + dhy * (d.node_y[vid[i]] - yc);
    if (hp[i] < kZero) adjust = true;
  }
  double gx, gy;
  if (adjust) {
    double zp[3], x[3], y[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      hp[i] = fmin2(kZero, hp[i]);
      zp[i] = d.zvtx[vid[i]] + hp[i];
      x[i] = d.node_x[vid[i]];
      y[i] = d.node_y[vid[i]];
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
__device__ __forceinline__ void bed_source(const Dev& d, const Geo<float>& G, int c, double h_c, double* s2,
                                           double* s3) {
  const int T = d.T;
  const float dhx = G.delh_x[c], dhy = G.delh_y[c];
  const double xc = d.xc[c], yc = d.yc[c];
  int vid[3];
  double hp[3];
  bool adjust = false;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    vid[i] = d.vert[(size_t)i * T + c];
    hp[i] = h_c + (double)(dhx * (float)(d.node_x[vid[i]] - xc) + dhy * (float)(d.node_y[vid[i]] - yc));
    if (hp[i] < kZero) adjust = true;
  }
  if (adjust) {
    double zp[3], x[3], y[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      zp[i] = d.zvtx[vid[i]] + fmin2(kZero, hp[i]);
      x[i] = d.node_x[vid[i]];
      y[i] = d.node_y[vid[i]];
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

// Fluxes, sources and the RK update of stage s (1-based) for cell c: the faces are
// added to phi in the order invisc_fluxes.f90 visits them (phi = zero first,
// solverFVT.f90:194), then the bed slope, then the RK update.  phi and the RK
// combination are FP64 on both paths.
template <class R>
__device__ __forceinline__ void assemble_phi(const Dev& d, const Geo<R>& G, int c, const double* __restrict__ hs,
                                             const uint8_t* __restrict__ dry, double* p1o, double* p2o, double* p3o) {
  const int T = d.T;
  const bool dry_c = dry[c];
  const double h_c = hs[c];
  double p1 = kZero, p2 = kZero, p3 = kZero;
  const uint8_t ord = d.forder[c];
  // Issue the loads of all three faces before the (ordered) accumulation: face
  // descriptors first, then the edge fluxes of the interior faces, so the gathers
  // overlap instead of forming one dependent chain per face.
  int fj[3], fkd[3], fre[3];
#pragma unroll
  for (int t = 0; t < 3; t++) {
    fj[t] = (ord >> (2 * t)) & 3;
    const size_t q = (size_t)fj[t] * T + c;
    fkd[t] = d.fkind[q] & 7;
    fre[t] = d.fref[q];
  }
  bool fok[3];
  R fv[3][3];
#pragma unroll
  for (int t = 0; t < 3; t++) {
    fok[t] = false;
    fv[t][0] = fv[t][1] = fv[t][2] = R(0);
    if (fkd[t] == FACE_LEFT || fkd[t] == FACE_RIGHT) {
      const int e = fre[t];  // flux*length of the edge, evaluated once by k_eflux
      fok[t] = d.eok[e];
      fv[t][0] = G.efx[e];
      fv[t][1] = G.efx[d.ne + e];
      fv[t][2] = G.efx[2 * d.ne + e];
    }
  }
#pragma unroll
  for (int t = 0; t < 3; t++) {
    const int j = fj[t];
    const size_t q = (size_t)j * T + c;
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
        const int w = fre[t];
        const double h1 = d.hvtx[d.wall_p1[w]], h2 = d.hvtx[d.wall_p2[w]];
        double hedge = qsqrt((h1 * h1 + h1 * h2 + h2 * h2) * kOneThird);
        if (hedge < kZero) hedge = kZero;
        if (hedge < d.h_dry) continue;
        p2 = p2 - kHalf * kG * hedge * hedge * nx * len;
        p3 = p3 - kHalf * kG * hedge * hedge * ny * len;
      } else {  // weslp2_fluxes.f90:34-76
        const size_t qc = (size_t)j * T + c;
        const double hleft = recon(h_c, G.delh_x[c], G.rc_x[qc], G.delh_y[c], G.rc_y[qc]);
        if (hleft < d.h_dry) continue;
        const double uleft = recon(d.u_b[c], G.delu_x[c], G.rc_x[qc], G.delu_y[c], G.rc_y[qc]);
        const double vleft = recon(d.v_b[c], G.delv_x[c], G.rc_x[qc], G.delv_y[c], G.rc_y[qc]);
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
      const int e = fre[t];
      p1 = p1 - d.bc_c[e];
      p2 = p2 - d.bc_c[d.nbce + e];
      p3 = p3 - d.bc_c[2 * d.nbce + e];
    }
  }
  if (!dry_c) {
    double s2, s3;
    bed_source(d, G, c, h_c, &s2, &s3);
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
                                          double p3, uint8_t* __restrict__ dry_next) {
  const int T = d.T;
  // RK update (solverFVT.f90:259-283)
  const double u_c = d.u_a[c], v_c = d.v_a[c];
  double delt;
  if (d.steady) {
    const double um = (h_c < d.h_dry) ? kZero : qsqrt(u_c * u_c + v_c * v_c);
    const double wc = dry_c ? kZero : sqrt(kG * h_c);
    delt = um + wc;
    if (delt < SMALL_F) delt = 1.044;
    delt = d.cfl * d.area[c] / (delt * d.perim[c]);
    if (s == d.K && c == d.sc[d.cell_sid[c]].last_cell) d.sc[d.cell_sid[c]].delt_fric = delt;
  } else {
    delt = d.sc[d.cell_sid[c]].delt;
  }
  const double dt = delt / d.area[c];
  double rh = kZero, ru = kZero, rv = kZero;
  for (int j = 0; j <= s - 1; j++) {
    // a zero coefficient (SSP-RK3 stage 3, level 1) adds a signed zero to a sum that
    // started at +0, which leaves its bits unchanged: skip the loads
    if (d.alpha[s][j] == kZero) continue;
    const size_t q = (size_t)j * T + c;
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
  const size_t qs = (size_t)s * T + c;
  d.rkh[qs] = rh;
  d.rku[qs] = ru;
  d.rkv[qs] = rv;
  d.u_a[c] = un;
  d.v_a[c] = vn;
  if (s < d.K) {
    double um;
    dry_next[c] = dry_flag(rh, un, vn, d.h_dry, d.h_wet, &um);
  } else {
    d.phimax[c] = fmax2(fmax2(fmax2(kZero, fabs(p1)), fabs(p2)), fabs(p3));
  }
}

template <class R>
__device__ __forceinline__ void flux_cell(const Dev& d, const Geo<R>& G, int s, int c, const double* __restrict__ hs,
                                          const uint8_t* __restrict__ dry, uint8_t* __restrict__ dry_next) {
  double p1, p2, p3;
  assemble_phi<R>(d, G, c, hs, dry, &p1, &p2, &p3);
  rk_update(d, s, c, hs[c], dry[c] != 0, p1, p2, p3, dry_next);
}

// Residual smoothing (solverFVT.f90:238-256, activateRSAVG): the stage's phi is
// assembled into d.phi (and its copy phi0), smoothed by Gauss-Seidel passes over the
// cells of one colour of the t2t stencil at a time (cells of a colour share no
// stencil edge, so each reads its neighbours' latest values exactly as a serial sweep
// in colour order does), then every cell is updated.
template <class R>
__global__ void __launch_bounds__(128) k_flux_phi(Dev d, Geo<R> G, const double* __restrict__ hs,
                                              const uint8_t* __restrict__ dry, int bc_cells) {
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
  const int sid = d.cell_sid[c];
  if (sid < 0 || d.sc[sid].converged) return;
  double p1, p2, p3;
  assemble_phi<R>(d, G, c, hs, dry, &p1, &p2, &p3);
  const size_t T = d.T;
  d.phi[c] = p1;
  d.phi[T + c] = p2;
  d.phi[2 * T + c] = p3;
  d.phi0[c] = p1;
  d.phi0[T + c] = p2;
  d.phi0[2 * T + c] = p3;
}

__global__ void __launch_bounds__(256) k_rsavg(Dev d, int off, int cnt) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= cnt) return;
  const int c = d.rs_cells[off + q];
  const int sid = d.cell_sid[c];
  if (sid < 0 || d.sc[sid].converged) return;
  const size_t T = d.T;
  const int n = d.nst[c];
  for (int k = 0; k < 3; k++) {
    double p = d.rs_fac1 * d.phi0[k * T + c];
    for (int m = 0; m < n; m++) p = p + d.rs_fac2 * d.phi[k * T + d.st_id[(size_t)m * T + c]];
    d.phi[k * T + c] = p;
  }
}

__global__ void __launch_bounds__(128) k_update(Dev d, int s, const double* __restrict__ hs,
                                            const uint8_t* __restrict__ dry, uint8_t* __restrict__ dry_next) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.T) return;
  const int sid = d.cell_sid[c];
  if (sid < 0 || d.sc[sid].converged) return;
  const size_t T = d.T;
  rk_update(d, s, c, hs[c], dry[c] != 0, d.phi[c], d.phi[T + c], d.phi[2 * T + c], dry_next);
}

// All cells without an open-boundary face (those wait for k_bc in k_flux_bc).
template <class R>
__global__ void __launch_bounds__(128, 10) k_flux(Dev d, Geo<R> G, int s, const double* __restrict__ hs,
                                              const uint8_t* __restrict__ dry, uint8_t* __restrict__ dry_next) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.T) return;
  const int sid = d.cell_sid[c];
  if (sid < 0 || d.sc[sid].converged) return;
  if (d.forder[c] & kOrderHasBc) return;
  flux_cell<R>(d, G, s, c, hs, dry, dry_next);
}

// The cells with an open-boundary face, after k_bc.
template <class R>
__global__ void __launch_bounds__(128) k_flux_bc(Dev d, Geo<R> G, int s, const double* __restrict__ hs,
                                                 const uint8_t* __restrict__ dry, uint8_t* __restrict__ dry_next) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.nbc_cells) return;
  const int c = d.bc_cells[i];
  if (d.sc[d.cell_sid[c]].converged) return;
  flux_cell<R>(d, G, s, c, hs, dry, dry_next);
}

// ---------------------------------------------------------------------------
// After the RK stages: find_dry_cells, fric_terms_impl, hvalve, rk level copy and the
// block partials of the iteration's reductions (solverFVT.f90:335-386, 407-445).
// kHalo: the handle links partitions, and halo cells stay out of the partials.
template <bool kHalo>
__global__ void __launch_bounds__(kRedThreads) k_fric(Dev d) {
  __shared__ double sm[kRedThreads / 32];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int T = d.T, K = d.K;
  const int sid = c < T ? d.cell_sid[c] : -1;
  // a block never spans two scenarios, so this test is uniform over the block
  if (d.sc[d.cell_sid[blockIdx.x * blockDim.x] < 0 ? 0 : d.cell_sid[blockIdx.x * blockDim.x]].converged) return;
  double st = kZero, sb = kZero, tm = kZero, rm = kZero, dtc = kVlarge;
  if (sid >= 0) {
    const size_t qk = (size_t)K * T + c;
    const double h = d.rkh[qk];
    double u = d.u_a[c], v = d.v_a[c];
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
          const size_t q = (size_t)j * T + c;
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
  double* pb = d.part + 8 * blockIdx.x;
  double r0 = block_sum<kRedThreads>(st, sm);
  if (threadIdx.x == 0) pb[0] = r0;
  double r1 = block_sum<kRedThreads>(sb, sm);
  if (threadIdx.x == 0) pb[1] = r1;
  double r2 = block_sum<kRedThreads>(tm, sm);
  if (threadIdx.x == 0) pb[2] = r2;
  double r3 = block_max<kRedThreads>(rm, sm);
  if (threadIdx.x == 0) pb[3] = r3;
  double r4 = block_min<kRedThreads>(dtc, sm);
  if (threadIdx.x == 0) pb[4] = r4;
}

__global__ void __launch_bounds__(kRedThreads) k_final(Dev d) {
  __shared__ double sm[kRedThreads / 32];
  const int sid = blockIdx.x;
  Scalars* sc = &d.sc[sid];
  if (sc->converged) return;
  double a0 = kZero, a1 = kZero, a2 = kZero, a3 = kZero, a4 = kVlarge;
  for (int b = threadIdx.x; b < sc->blk_cnt; b += blockDim.x) {
    const double* pb = d.part + 8 * (sc->blk_off + b);
    a0 = a0 + pb[0];
    a1 = a1 + pb[1];
    a2 = a2 + pb[2];
    a3 = fmax2(a3, pb[3]);
    a4 = fmin2(a4, pb[4]);
  }
  const double sumtop = block_sum<kRedThreads>(a0, sm);
  const double sumbot = block_sum<kRedThreads>(a1, sm);
  const double tmass = block_sum<kRedThreads>(a2, sm);
  const double rmax_phi = block_max<kRedThreads>(a3, sm);
  const double dtmin = block_min<kRedThreads>(a4, sm);
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

// ---------------------------------------------------------------------------
// The output pass of solverFVT.f90:389-405 (to_vertices.f90:26-65, ctr2vtx.f90:69-80,
// wetdryvfix.f90, enforce_bcs.f90:37-171, vbc_by_h.f90, error_est.f90 etype 2) after
// an iteration.  The depths come from zeta of the last stage's start (solverFVT.f90:169
// is the only assignment of zeta) and the dry flags of the find_dry_cells call before
// the friction step (:335), as in the reference.

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

// enforce_bcs.f90:124-169 with vbc_by_h.f90 for one inflow string, serial in node order
// as the reference (the sums of vbc_by_h keep their order)
__device__ void out_inflow_string(const Dev& d, const OutputArgs& a, int b) {
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
  if (threadIdx.x == 0) d.part[8 * blockIdx.x + 4] = r;
}
__global__ void __launch_bounds__(kRedThreads) k_out_dtfinal(Dev d) {
  __shared__ double sm[kRedThreads / 32];
  Scalars* sc = &d.sc[blockIdx.x];
  double a4 = kVlarge;
  for (int b = threadIdx.x; b < sc->blk_cnt; b += blockDim.x) a4 = fmin2(a4, d.part[8 * (sc->blk_off + b) + 4]);
  const double dtmin = block_min<kRedThreads>(a4, sm);
  if (threadIdx.x == 0) sc->delt = dtmin;
}

void launch_output(const Dev& d, const Geo<double>& Gd, const Geo<float>& Gf, bool mixed, const OutputArgs& a,
                   cudaStream_t st) {
  const int gN = (d.N + 255) / 256, gT = (d.T + 255) / 256;
  k_out_depth<<<gN, 256, 0, st>>>(d, a);
  if (mixed) k_out_cell<float><<<gT, 256, 0, st>>>(d, Gf, a);
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

void launch_halo(const Dev& d, int level, uint8_t* f1, uint8_t* f2, cudaStream_t st) {
  k_halo<<<(d.nhalo + 255) / 256, 256, 0, st>>>(d, level, f1, f2);
}
void launch_link_fric(const Dev& d, cudaStream_t st) { k_link_fric<<<1, 32, 0, st>>>(d); }
void launch_fric(const Dev& d, cudaStream_t st) {
  if (d.nhalo > 0) k_fric<true><<<d.nblk_red, kRedThreads, 0, st>>>(d);
  else k_fric<false><<<d.nblk_red, kRedThreads, 0, st>>>(d);
}
void launch_link_dt(const Dev& d, cudaStream_t st) { k_link_dt<<<1, 32, 0, st>>>(d); }
void launch_link(const Dev& d, cudaStream_t st) { k_link<<<1, 32, 0, st>>>(d); }

// ---------------------------------------------------------------------------
// Host launchers of the templated stage kernels (api.cu is not templated).
template <class R>
static void launch_stage_t(const StageLaunch& L, const Dev& d, const Geo<R>& G) {
  switch (L.which) {
    case STAGE_GRAD:
      k_grad<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry, L.rku_prev, L.rkv_prev);
      break;
    case STAGE_BC:
      k_bc<R><<<L.grid, L.block, L.smem, L.stream>>>(d, G, L.hs, L.dry);
      break;
    case STAGE_EFLUX:
      k_eflux<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry);
      break;
    case STAGE_FLUX:
      k_flux<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.s, L.hs, L.dry, L.dry_next);
      break;
    case STAGE_FLUX_BC:
      k_flux_bc<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.s, L.hs, L.dry, L.dry_next);
      break;
    case STAGE_PHI:
      k_flux_phi<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry, 0);
      break;
    case STAGE_PHI_BC:
      k_flux_phi<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry, 1);
      break;
    case STAGE_UPDATE:
      k_update<<<L.grid, L.block, 0, L.stream>>>(d, L.s, L.hs, L.dry, L.dry_next);
      break;
    case STAGE_CULVERT:
      k_culvert<R><<<L.grid, L.block, 0, L.stream>>>(d, G, L.hs, L.dry);
      break;
  }
}

void launch_stage(const StageLaunch& L, const Dev& d, const Geo<double>& Gd, const Geo<float>& Gf, bool mixed) {
  if (mixed) launch_stage_t<float>(L, d, Gf);
  else launch_stage_t<double>(L, d, Gd);
}

void launch_rsavg(const Dev& d, int off, int cnt, cudaStream_t st) {
  if (cnt > 0) k_rsavg<<<(cnt + 255) / 256, 256, 0, st>>>(d, off, cnt);
}

void set_bc_smem_limit(int bytes) {
  cudaFuncSetAttribute(k_bc<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_bc<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace storm
