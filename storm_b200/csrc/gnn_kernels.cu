// gnn_kernels.cu -- warm-start network on the cell-dual graph: fused two-layer MLP
// kernels on the sm_100a tensor cores (tcgen05 MMA, TMEM accumulators), their
// backward passes, and the gather/scatter, loss and optimiser kernels around them.
//
// The network has no counterpart in the reference (SToRM starts steady runs from the
// user's initial condition); it predicts an initial h, hu, hv for the solver, which
// then runs on to its own stop test.
//
// Graph layout.  Cells are padded to Tp (a multiple of 128).  Every cell c owns three
// directed edge rows, one per local face k: row k*Tp + c carries the message from the
// neighbour nbr[k*Tp + c] (-1: no neighbour) into c.  An MLP input row is the
// concatenation of up to three 128-wide segments, each read from a bf16 matrix
// through an optional row map, or summed over the three edge rows of a cell
// (the message aggregation), so the edge update [e, h_src, h_dst] and the node
// update [h, sum_k e_k] need no materialised concatenation.
//
// One CTA (256 threads) works on tiles of 128 rows.  Forward: D1 = A W1^T over the
// segments (two staging buffers so a segment's load overlaps the previous segment's
// MMAs), epilogue bias+ReLU into a shared-memory tile, D2 = a1 W2^T, epilogue
// bias (+ residual).  Weights stay resident in shared memory for the CTA's lifetime.
#include <cstdint>
#include <cstdio>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "umma.cuh"

namespace storm {
namespace gnn {

using bf16 = __nv_bfloat16;

constexpr int kRows = 128;     // rows per tile (MMA M)
constexpr int kHid = 128;      // hidden width
constexpr int kThreads = 256;  // 8 warps
constexpr int kMaxSeg = 3;

struct Seg {
  const bf16* src;       // [*, width] row-major
  const int32_t* idx;    // row map (nullptr: identity); a negative entry reads zeros
  int32_t width;         // 64 or 128
  int32_t agg;           // 1: sum of rows r + k*agg_stride (k < 3) whose nbr entry is >= 0
  int32_t agg_stride;
  const int32_t* nbr;    // [3*agg_stride] neighbour table (mask of the aggregation)
};

struct MlpFwd {
  int32_t rows, nseg, k_in, n_out;
  Seg seg[kMaxSeg];
  const bf16* w1;   // [128][k_in]
  const float* b1;  // [128]
  const bf16* w2;   // [n_out][128]
  const float* b2;  // [n_out]
  const bf16* res;  // [rows][n_out] residual added to the output, or nullptr
  bf16* out;        // [rows][n_out]
  float* out_f32;   // optional fp32 copy of the output
  bf16* a1_save;    // [rows][128] hidden activation (training), or nullptr
  int32_t* err;
};

// Backward, data part: da1 = dy W2, dz1 = da1 * (a1 > 0), dA = dz1 W1 split per segment.
struct SegGrad {
  float* out;         // [rows][width] fp32, or nullptr (segment gradient not needed)
  const float* add;   // added to the result (the residual path), or nullptr
};
struct MlpBwdData {
  int32_t rows, nseg, k_in, n_out;
  int32_t seg_width[kMaxSeg];
  SegGrad dseg[kMaxSeg];
  const float* dy;    // [rows][n_out]
  const bf16* a1;     // [rows][128]
  const bf16* w1;     // [128][k_in]
  const bf16* w2;     // [n_out][128]
  bf16* dz1_save;     // [rows][128]
  int32_t* err;
};

// Backward, weight part: per-CTA partial dW1 = dz1^T A, dW2 = dy^T a1, db1, db2.
struct MlpBwdWeight {
  int32_t rows, nseg, k_in, n_out;
  Seg seg[kMaxSeg];
  const float* dy;    // [rows][n_out]
  const bf16* a1;     // [rows][128]
  const bf16* dz1;    // [rows][128]
  float* part;        // [grid][128*k_in + 128 + n_out*128 + n_out]
  int32_t* err;
};

__device__ __forceinline__ void set_err(int32_t* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// ---- shared-memory staging -------------------------------------------------------

// The staging helpers below give every thread up to eight 16-byte chunks of the tile
// (chunk q = threadIdx.x + i*256) and issue all of a thread's global loads before any
// of its shared-memory stores, so 32 KB per SM are in flight instead of one load per
// thread at a time.
constexpr int kChunksPerThread = 8;  // 128 rows x 16 chunks / 256 threads

__device__ __forceinline__ void store_chunk(uint8_t* dst, int q, int cpr, uint4 v) {
  const int r = q / cpr, c = q - r * cpr;
  const int blk = c >> 3;
  *reinterpret_cast<uint4*>(dst + blk * (kRows * 128) + umma::sw128_offset(r, (c & 7) * 8)) = v;
}

template <int R>
__device__ __forceinline__ void stage_agg_rounds(const Seg& s, int row0, uint8_t* dst, int tid, int nthr, int cpr,
                                                 int total) {
  for (int h = 0; h * nthr < total; h += R) {
    uint4 w[R][3];
    bool m[R][3];
#pragma unroll
    for (int i = 0; i < R; i++) {
      const int q = tid + (h + i) * nthr;
      const int row = row0 + q / cpr;
#pragma unroll
      for (int k = 0; k < 3; k++)
        m[i][k] = (q < total) && s.nbr[static_cast<size_t>(k) * s.agg_stride + row] >= 0;
    }
#pragma unroll
    for (int i = 0; i < R; i++) {
      const int q = tid + (h + i) * nthr;
      const int row = row0 + q / cpr, c = q % cpr;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        w[i][k] = make_uint4(0, 0, 0, 0);
        if (m[i][k]) {
          const size_t er = static_cast<size_t>(k) * s.agg_stride + row;
          w[i][k] = *reinterpret_cast<const uint4*>(s.src + er * s.width + c * 8);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < R; i++) {
      const int q = tid + (h + i) * nthr;
      if (q >= total) continue;
      float acc[8];
#pragma unroll
      for (int j = 0; j < 8; j++) acc[j] = 0.f;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        if (!m[i][k]) continue;
        const bf16* b = reinterpret_cast<const bf16*>(&w[i][k]);
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += __bfloat162float(b[j]);
      }
      uint4 v;
      bf16* o = reinterpret_cast<bf16*>(&v);
#pragma unroll
      for (int j = 0; j < 8; j++) o[j] = __float2bfloat16(acc[j]);
      store_chunk(dst, q, cpr, v);
    }
  }
}

// Stage rows [row0, row0+128) of one segment into `dst` (blocks of 128 x 64, 16 KB
// each) with `nthr` threads (thread `tid` of them), in rounds of eight chunks per thread.
__device__ __forceinline__ void stage_segment(const Seg& s, int row0, uint8_t* dst, int tid = -1,
                                              int nthr = kThreads) {
  if (tid < 0) tid = threadIdx.x;
  const int cpr = s.width >> 3;  // 16-byte chunks per row
  const int total = kRows * cpr;
  if (!s.agg) {
    for (int q0 = 0; q0 < total; q0 += kChunksPerThread * nthr) {
      uint4 v[kChunksPerThread];
      int srow[kChunksPerThread];
#pragma unroll
      for (int i = 0; i < kChunksPerThread; i++) {
        const int q = q0 + tid + i * nthr;
        const int row = row0 + q / cpr;
        srow[i] = (q < total) ? (s.idx ? s.idx[row] : row) : -1;
      }
#pragma unroll
      for (int i = 0; i < kChunksPerThread; i++) {
        const int q = q0 + tid + i * nthr;
        const int c = q % cpr;
        v[i] = make_uint4(0, 0, 0, 0);
        if (srow[i] >= 0)
          v[i] = *reinterpret_cast<const uint4*>(s.src + static_cast<size_t>(srow[i]) * s.width + c * 8);
      }
#pragma unroll
      for (int i = 0; i < kChunksPerThread; i++) {
        const int q = q0 + tid + i * nthr;
        if (q < total) store_chunk(dst, q, cpr, v[i]);
      }
    }
    return;
  }
  // aggregation: sum of the three edge rows of each cell, in rounds of eight chunks
  // per thread (24 loads in flight) for the forward kernel's producers, four otherwise
  if (nthr <= 224) stage_agg_rounds<8>(s, row0, dst, tid, nthr, cpr, total);
  else stage_agg_rounds<4>(s, row0, dst, tid, nthr, cpr, total);
}

// Stage an fp32 [rows][width] tile as bf16 (width 64 or 128).
__device__ __forceinline__ void stage_f32(const float* src, int width, int row0, uint8_t* dst) {
  const int cpr = width >> 3;
  const int total = kRows * cpr;
#pragma unroll
  for (int h = 0; h < kChunksPerThread; h += 4) {
    float4 a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int q = threadIdx.x + (h + i) * kThreads;
      a[i] = b[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (q < total) {
        const int r = q / cpr, c = q - r * cpr;
        const float4* p = reinterpret_cast<const float4*>(src + static_cast<size_t>(row0 + r) * width + c * 8);
        a[i] = p[0];
        b[i] = p[1];
      }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int q = threadIdx.x + (h + i) * kThreads;
      if (q >= total) continue;
      uint4 v;
      bf16* o = reinterpret_cast<bf16*>(&v);
      o[0] = __float2bfloat16(a[i].x); o[1] = __float2bfloat16(a[i].y); o[2] = __float2bfloat16(a[i].z);
      o[3] = __float2bfloat16(a[i].w); o[4] = __float2bfloat16(b[i].x); o[5] = __float2bfloat16(b[i].y);
      o[6] = __float2bfloat16(b[i].z); o[7] = __float2bfloat16(b[i].w);
      store_chunk(dst, q, cpr, v);
    }
  }
}

// Stage a bf16 row-major [nrows][ncols] matrix (ncols multiple of 64) as blocks of
// nrows x 64 (block stride nrows*128 bytes); loads batched eight per thread.
__device__ __forceinline__ void stage_matrix(const bf16* src, int nrows, int ncols, uint8_t* dst) {
  const int cpr = ncols >> 3;
  const int total = nrows * cpr;
  for (int q0 = 0; q0 < total; q0 += kChunksPerThread * kThreads) {
    uint4 v[kChunksPerThread];
#pragma unroll
    for (int i = 0; i < kChunksPerThread; i++) {
      const int q = q0 + threadIdx.x + i * kThreads;
      v[i] = make_uint4(0, 0, 0, 0);
      if (q < total) {
        const int r = q / cpr, c = q - r * cpr;
        v[i] = *reinterpret_cast<const uint4*>(src + static_cast<size_t>(r) * ncols + c * 8);
      }
    }
#pragma unroll
    for (int i = 0; i < kChunksPerThread; i++) {
      const int q = q0 + threadIdx.x + i * kThreads;
      if (q < total) {
        const int r = q / cpr, c = q - r * cpr;
        const int blk = c >> 3;
        *reinterpret_cast<uint4*>(dst + blk * (nrows * 128) + umma::sw128_offset(r, (c & 7) * 8)) = v[i];
      }
    }
  }
}

constexpr int kProducersAsync = 352;

// Asynchronous copy of one 16-byte chunk global -> shared (zero-filled when `valid` is
// false); the copies of a thread are grouped with commit / wait_group.
__device__ __forceinline__ void cp_async16(uint8_t* dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(umma::smem_addr(dst)), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Issue (without waiting) the copies of one gathered, non-aggregated segment tile by
// the 352 producer threads: every thread resolves the source rows of its (at most 6)
// chunks first, all index loads in flight together, then issues its copies.
constexpr int kMaxAsyncChunks = (kRows * 16 + kProducersAsync - 1) / kProducersAsync;  // 128 x 16 chunks
__device__ __forceinline__ void stage_segment_async(const Seg& s, int row0, uint8_t* dst, int tid) {
  const int cpr = s.width >> 3;
  const int total = kRows * cpr;
  int srow[kMaxAsyncChunks];
#pragma unroll
  for (int i = 0; i < kMaxAsyncChunks; i++) {
    const int q = tid + i * kProducersAsync;
    const int row = row0 + q / cpr;
    srow[i] = (q < total) ? (s.idx ? s.idx[row] : row) : -1;
  }
#pragma unroll
  for (int i = 0; i < kMaxAsyncChunks; i++) {
    const int q = tid + i * kProducersAsync;
    if (q >= total) continue;
    const int r = q / cpr, c = q - r * cpr;
    const bf16* src = s.src + static_cast<size_t>(srow[i] >= 0 ? srow[i] : 0) * s.width + c * 8;
    cp_async16(dst + (c >> 3) * (kRows * 128) + umma::sw128_offset(r, (c & 7) * 8), src, srow[i] >= 0);
  }
}

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~static_cast<uintptr_t>(1023));
}

// Issue D (+)= A B^T over K (multiple of 16), A and B K-major tiles with blocks of 64
// columns: a_blk / b_blk are the byte strides between their 64-column blocks.
__device__ __forceinline__ void mma_kmajor(uint32_t tmem_d, uint32_t a, uint32_t a_blk, uint32_t b,
                                           uint32_t b_blk, int K, uint32_t idesc, bool accumulate) {
  for (int k = 0; k < K; k += 16) {
    const uint32_t off = (k & 63) * 2;
    const uint64_t ad = umma::desc_kmajor(a + (k >> 6) * a_blk + off);
    const uint64_t bd = umma::desc_kmajor(b + (k >> 6) * b_blk + off);
    umma::mma_bf16(tmem_d, ad, bd, idesc, (accumulate || k > 0) ? 1u : 0u);
  }
}

// ---- forward ----------------------------------------------------------------------

// Shared memory: W1 (128 x k_in), W2 (n_out x 128), two A staging buffers (128 x 128),
// the hidden tile (128 x 128), barriers.
__host__ __device__ constexpr size_t fwd_smem_bytes(int k_in, int n_out) {
  return 1024 + static_cast<size_t>(kHid) * k_in * 2 + static_cast<size_t>(n_out) * kHid * 2 +
         2 * (kRows * 128 * 2) + kRows * kHid * 2 + 256;
}

// Warp roles of the forward kernel (512 threads, sixteen warps, so up to 128
// registers each):
//   warps 0-10  producers: gather each input segment of the CTA's tiles into the
//               two-buffer staging ring (a buffer is refilled once the MMAs that read
//               it have completed); the gathers of scattered rows are what bounds the
//               kernel, so most warps do them;
//   warps 11-14 epilogue: TMEM -> bias + ReLU -> hidden tile, then TMEM -> bias
//               (+ residual) -> output; warp w reads TMEM lanes 32(w%4)..32(w%4)+31;
//   warp 15     one thread issues the MMAs: D1[slot] = A W1^T over the segments, then
//               D2[slot] = a1 W2^T once the epilogue has written the hidden tile.
// D1 and D2 are double-buffered in TMEM (slot = tile parity), so the MMAs of tile t+1
// proceed while the epilogue drains tile t.  Every wait is bounded; a wait that runs
// out raises the abort flag, which every role polls.
constexpr int kFwdThreads = 512;
__device__ __forceinline__ bool aborted(const int* flag) { return *reinterpret_cast<const volatile int*>(flag) != 0; }
constexpr int kProducers = 352;

__global__ void __launch_bounds__(kFwdThreads, 1) k_mlp_fwd(MlpFwd p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = align1024(smem_raw);
  uint8_t* w1s = base;
  uint8_t* w2s = w1s + kHid * p.k_in * 2;
  uint8_t* abuf = w2s + p.n_out * kHid * 2;  // 2 x 32 KB
  uint8_t* a1s = abuf + 2 * (kRows * 128 * 2);
  uint64_t* bars = reinterpret_cast<uint64_t*>(a1s + kRows * kHid * 2);
  uint64_t* full = bars;        // [2] staging buffer filled (one arrival per producer)
  uint64_t* empty = bars + 2;   // [2] MMAs reading the buffer done (commit)
  uint64_t* d1full = bars + 4;  // [2] D1[slot] complete (commit)
  uint64_t* a1full = bars + 6;  // hidden tile written (128 epilogue arrivals)
  uint64_t* d2full = bars + 7;  // [2] D2[slot] complete (commit)
  uint64_t* tfree = bars + 9;   // [2] epilogue done with D1/D2[slot] (128 arrivals)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 11);
  __shared__ int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    umma::mbar_init(&full[0], kProducers);
    umma::mbar_init(&full[1], kProducers);
    umma::mbar_init(&empty[0], 1);
    umma::mbar_init(&empty[1], 1);
    umma::mbar_init(&d1full[0], 1);
    umma::mbar_init(&d1full[1], 1);
    umma::mbar_init(a1full, kRows);
    umma::mbar_init(&d2full[0], 1);
    umma::mbar_init(&d2full[1], 1);
    umma::mbar_init(&tfree[0], kRows);
    umma::mbar_init(&tfree[1], kRows);
    umma::mbar_fence_init();
    s_abort = 0;
  }
  if (warp == 0) umma::tmem_alloc(tmem_slot, 512);
  {  // weights, staged by all threads
    const int cpr1 = p.k_in >> 3, tot1 = kHid * cpr1;
    for (int q = threadIdx.x; q < tot1; q += kFwdThreads) {
      const int r = q / cpr1, c = q - r * cpr1;
      *reinterpret_cast<uint4*>(w1s + (c >> 3) * (kHid * 128) + umma::sw128_offset(r, (c & 7) * 8)) =
          *reinterpret_cast<const uint4*>(p.w1 + static_cast<size_t>(r) * p.k_in + c * 8);
    }
    const int cpr2 = kHid >> 3, tot2 = p.n_out * cpr2;
    for (int q = threadIdx.x; q < tot2; q += kFwdThreads) {
      const int r = q / cpr2, c = q - r * cpr2;
      *reinterpret_cast<uint4*>(w2s + (c >> 3) * (p.n_out * 128) + umma::sw128_offset(r, (c & 7) * 8)) =
          *reinterpret_cast<const uint4*>(p.w2 + static_cast<size_t>(r) * kHid + c * 8);
    }
  }
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const int ntiles = p.rows / kRows;

  if (warp < 11) {
    // ---- producers
    // Gathered segments are copied with cp.async, keeping the copies of two segments
    // in flight (a segment is announced once the next one has been issued); the
    // aggregation segment sums three rows in registers.
    const int tid = threadIdx.x;
    uint32_t g = 0;
    int pending = -1;  // buffer whose cp.async copies are issued but not yet announced
    for (int tile = blockIdx.x; tile < ntiles && !aborted(&s_abort); tile += gridDim.x) {
      for (int s = 0; s < p.nseg; s++, g++) {
        const int b = g & 1;
        if (g >= 2 && !umma::mbar_wait(&empty[b], ((g >> 1) - 1) & 1)) {
          s_abort = 1;
          break;
        }
        uint8_t* dst = abuf + b * (kRows * 128 * 2);
        if (p.seg[s].agg) {
          if (pending >= 0) {
            cp_async_wait<0>();
            umma::fence_async_smem();
            umma::mbar_arrive(&full[pending]);
            pending = -1;
          }
          stage_segment(p.seg[s], tile * kRows, dst, tid, kProducers);
          umma::fence_async_smem();
          umma::mbar_arrive(&full[b]);
        } else {
          stage_segment_async(p.seg[s], tile * kRows, dst, tid);
          cp_async_commit();
          if (pending >= 0) {
            cp_async_wait<1>();
            umma::fence_async_smem();
            umma::mbar_arrive(&full[pending]);
          }
          pending = b;
        }
      }
    }
    if (pending >= 0) {
      cp_async_wait<0>();
      umma::fence_async_smem();
      umma::mbar_arrive(&full[pending]);
    }
  } else if (warp < 15) {
    // ---- epilogue
    const int q = warp & 3;
    const int r = q * 32 + lane;  // row of the tile = TMEM lane
    const uint32_t lane_off = static_cast<uint32_t>(q * 32) << 16;
    uint32_t t = 0;
    for (int tile = blockIdx.x; tile < ntiles && !aborted(&s_abort); tile += gridDim.x, t++) {
      const int slot = t & 1;
      const uint32_t d1 = tmem + slot * 128, d2 = tmem + 256 + slot * 128;
      const size_t row = static_cast<size_t>(tile) * kRows + r;
      if (!umma::mbar_wait(&d1full[slot], (t >> 1) & 1)) {
        s_abort = 1;
        break;
      }
      umma::fence_after_sync();
      for (int col0 = 0; col0 < kHid; col0 += 32) {
        float v[32];
        umma::tmem_ld32(d1 + lane_off + col0, v);
        uint4 pk[4];
        bf16* o = reinterpret_cast<bf16*>(pk);
#pragma unroll
        for (int j = 0; j < 32; j++) o[j] = __float2bfloat16(fmaxf(v[j] + p.b1[col0 + j], 0.f));
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int c = col0 + j * 8;
          *reinterpret_cast<uint4*>(a1s + (c >> 6) * (kRows * 128) + umma::sw128_offset(r, c & 63)) = pk[j];
          if (p.a1_save) *reinterpret_cast<uint4*>(p.a1_save + row * kHid + c) = pk[j];
        }
      }
      umma::fence_async_smem();
      umma::fence_before_sync();
      umma::mbar_arrive(a1full);
      if (!umma::mbar_wait(&d2full[slot], (t >> 1) & 1)) {
        s_abort = 1;
        break;
      }
      umma::fence_after_sync();
      for (int col0 = 0; col0 < p.n_out; col0 += 32) {
        float v[32];
        const size_t o0 = row * p.n_out + col0;
        if (p.res) {
          uint4 rr[4];
          const uint4* rp = reinterpret_cast<const uint4*>(p.res + o0);
#pragma unroll
          for (int j = 0; j < 4; j++) rr[j] = rp[j];
          umma::tmem_ld32(d2 + lane_off + col0, v);
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const bf16* b = reinterpret_cast<const bf16*>(&rr[j]);
#pragma unroll
            for (int u = 0; u < 8; u++) v[j * 8 + u] += __bfloat162float(b[u]);
          }
        } else {
          umma::tmem_ld32(d2 + lane_off + col0, v);
        }
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] += p.b2[col0 + j];
        uint4 pk[4];
        bf16* o = reinterpret_cast<bf16*>(pk);
#pragma unroll
        for (int j = 0; j < 32; j++) o[j] = __float2bfloat16(v[j]);
        uint4* op = reinterpret_cast<uint4*>(p.out + o0);
#pragma unroll
        for (int j = 0; j < 4; j++) op[j] = pk[j];
        if (p.out_f32) {
          float4* fp = reinterpret_cast<float4*>(p.out_f32 + o0);
#pragma unroll
          for (int j = 0; j < 8; j++) fp[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        }
      }
      umma::fence_before_sync();
      umma::mbar_arrive(&tfree[slot]);
    }
  } else if (lane == 0) {
    // ---- MMA issuer
    const uint32_t w1a = umma::smem_addr(w1s), w2a = umma::smem_addr(w2s);
    const uint32_t a1a = umma::smem_addr(a1s);
    const uint32_t idesc1 = umma::idesc_bf16(kRows, kHid, false, false);
    const uint32_t idesc2 = umma::idesc_bf16(kRows, p.n_out, false, false);
    uint32_t g = 0, t = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, t++) {
      const int slot = t & 1;
      const uint32_t d1 = tmem + slot * 128, d2 = tmem + 256 + slot * 128;
      if (t >= 2 && !umma::mbar_wait(&tfree[slot], ((t >> 1) - 1) & 1)) ok = false;
      int kcol = 0;
      for (int s = 0; s < p.nseg && ok; s++, g++) {
        const int b = g & 1;
        if (!umma::mbar_wait(&full[b], (g >> 1) & 1)) {
          ok = false;
          break;
        }
        umma::fence_after_sync();
        mma_kmajor(d1, umma::smem_addr(abuf + b * (kRows * 128 * 2)), kRows * 128,
                   w1a + (kcol >> 6) * (kHid * 128), kHid * 128, p.seg[s].width, idesc1, s > 0);
        umma::commit(&empty[b]);
        kcol += p.seg[s].width;
      }
      if (!ok) break;
      umma::commit(&d1full[slot]);
      if (!umma::mbar_wait(a1full, t & 1)) {
        ok = false;
        break;
      }
      umma::fence_after_sync();
      mma_kmajor(d2, a1a, kRows * 128, w2a, p.n_out * 128, kHid, idesc2, false);
      umma::commit(&d2full[slot]);
    }
    // drain: the last arrivals on the staging barriers before shared memory is released
    if (ok && g > 0) {
      const uint32_t uses0 = (g + 1) >> 1, uses1 = g >> 1;
      if (uses0 > 0 && !umma::mbar_wait(&empty[0], (uses0 - 1) & 1)) ok = false;
      if (uses1 > 0 && !umma::mbar_wait(&empty[1], (uses1 - 1) & 1)) ok = false;
    }
    if (t > 0 && ok) {  // the last D2 of each slot (the epilogue waited for them too)
      const uint32_t last = t - 1;
      if (!umma::mbar_wait(&d2full[last & 1], (last >> 1) & 1)) ok = false;
    }
    if (!ok) s_abort = 1;
  }
  umma::fence_before_sync();
  __syncthreads();
  if (s_abort && threadIdx.x == 0) set_err(p.err, 1);
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, 512);
  }
}

// ---- backward: data gradients -------------------------------------------------------

__host__ __device__ constexpr size_t bwd_data_smem_bytes(int k_in, int n_out) {
  return 1024 + static_cast<size_t>(kHid) * k_in * 2 + static_cast<size_t>(n_out) * kHid * 2 +
         kRows * 128 * 2 /* dy (up to 128 columns) */ + kRows * kHid * 2 /* dz1 */ + 256;
}

__global__ void __launch_bounds__(kThreads, 1) k_mlp_bwd_data(MlpBwdData p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = align1024(smem_raw);
  uint8_t* w1s = base;                                // [128 hid][k_in] blocks of 64 cols (16 KB)
  uint8_t* w2s = w1s + kHid * p.k_in * 2;             // [n_out][128]   blocks of 64 cols
  uint8_t* dys = w2s + p.n_out * kHid * 2;            // [128][n_out]
  uint8_t* dzs = dys + kRows * 128 * 2;               // [128][128]
  uint64_t* bars = reinterpret_cast<uint64_t*>(dzs + kRows * kHid * 2);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  __shared__ int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool need_da = false;
  for (int s = 0; s < p.nseg; s++) need_da |= (p.dseg[s].out != nullptr);
  if (threadIdx.x == 0) {
    umma::mbar_init(&bars[0], 1);
    umma::mbar_init(&bars[1], 1);
    umma::mbar_fence_init();
    s_abort = 0;
  }
  if (warp == 0) umma::tmem_alloc(tmem_slot, 512);
  stage_matrix(p.w1, kHid, p.k_in, w1s);
  stage_matrix(p.w2, p.n_out, kHid, w2s);
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t dda1 = tmem, dda = tmem + 128;
  const uint32_t w1a = umma::smem_addr(w1s), w2a = umma::smem_addr(w2s);
  const uint32_t dya = umma::smem_addr(dys), dza = umma::smem_addr(dzs);
  // da1 = dy W2 : A = dy [128 x n_out] K-major, B = W2 viewed [N=128 hid x K=n_out] MN-major
  const uint32_t idesc_a1 = umma::idesc_bf16(kRows, kHid, false, true);
  // dA = dz1 W1 : A = dz1 [128 x 128] K-major, B = W1 viewed [N=k_in x K=128] MN-major
  const int nchunk = p.k_in >= 128 ? 128 : p.k_in;
  const uint32_t idesc_da = umma::idesc_bf16(kRows, nchunk, false, true);

  const int ntiles = p.rows / kRows;
  const int lane_base = (warp & 3) * 32;
  const int r = lane_base + lane;
  const int half = warp >> 2;
  uint32_t it = 0;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
    const int row0 = tile * kRows;
    stage_f32(p.dy, p.n_out, row0, dys);
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
      // K = n_out rows of W2; K-step 16 advances dy by 32 bytes (inside a 64-col block)
      // and the MN-major W2 view by 16 rows (2 KB).
      for (int k = 0; k < p.n_out; k += 16) {
        const uint64_t ad = umma::desc_kmajor(dya + (k >> 6) * (kRows * 128) + (k & 63) * 2);
        const uint64_t bd = umma::desc_mnmajor(w2a + k * 128, p.n_out * 128);
        umma::mma_bf16(dda1, ad, bd, idesc_a1, k > 0 ? 1u : 0u);
      }
      umma::commit(&bars[0]);
    }
    if (!umma::mbar_wait(&bars[0], it & 1)) s_abort = 1;
    __syncthreads();
    if (s_abort) break;
    umma::fence_after_sync();
    // epilogue: dz1 = da1 * (a1 > 0)
    for (int cc = 0; cc < 64; cc += 32) {
      const int col0 = half * 64 + cc;
      float v[32];
      umma::tmem_ld32(dda1 + (static_cast<uint32_t>(lane_base) << 16) + col0, v);
      const uint4* ap = reinterpret_cast<const uint4*>(p.a1 + static_cast<size_t>(row0 + r) * kHid + col0);
      uint4 pk[4];
      bf16* o = reinterpret_cast<bf16*>(pk);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint4 w = ap[j];
        const bf16* b = reinterpret_cast<const bf16*>(&w);
#pragma unroll
        for (int t = 0; t < 8; t++) o[j * 8 + t] = __float2bfloat16(__bfloat162float(b[t]) > 0.f ? v[j * 8 + t] : 0.f);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int c = col0 + j * 8;
        *reinterpret_cast<uint4*>(dzs + (c >> 6) * (kRows * 128) + umma::sw128_offset(r, c & 63)) = pk[j];
        if (p.dz1_save)
          *reinterpret_cast<uint4*>(p.dz1_save + static_cast<size_t>(row0 + r) * kHid + c) = pk[j];
      }
    }
    if (!need_da) {
      umma::fence_before_sync();
      __syncthreads();
      continue;
    }
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
      for (int n0 = 0; n0 < p.k_in; n0 += nchunk) {
        for (int k = 0; k < kHid; k += 16) {
          const uint64_t ad = umma::desc_kmajor(dza + (k >> 6) * (kRows * 128) + (k & 63) * 2);
          // W1 rows k.. (K index = hid), columns n0.. (block n0/64 of 16 KB)
          const uint64_t bd = umma::desc_mnmajor(w1a + (n0 >> 6) * (kHid * 128) + k * 128, kHid * 128);
          umma::mma_bf16(dda + n0, ad, bd, idesc_da, k > 0 ? 1u : 0u);
        }
      }
      umma::commit(&bars[1]);
    }
    if (!umma::mbar_wait(&bars[1], it & 1)) s_abort = 1;
    __syncthreads();
    if (s_abort) break;
    umma::fence_after_sync();
    // epilogue: segment gradients (fp32), plus the residual-path addend
    {
      int kcol = 0;
      for (int s = 0; s < p.nseg; s++) {
        const int w = p.seg_width[s];
        const SegGrad g = p.dseg[s];
        if (g.out) {
          const int per_half = w / 2;
          for (int cc = 0; cc < per_half; cc += 32) {
            const int col0 = half * per_half + cc;
            float v[32];
            umma::tmem_ld32(dda + (static_cast<uint32_t>(lane_base) << 16) + kcol + col0, v);
            const size_t o0 = static_cast<size_t>(row0 + r) * w + col0;
            if (g.add) {
              const float4* ap = reinterpret_cast<const float4*>(g.add + o0);
#pragma unroll
              for (int j = 0; j < 8; j++) {
                const float4 a = ap[j];
                v[4 * j] += a.x; v[4 * j + 1] += a.y; v[4 * j + 2] += a.z; v[4 * j + 3] += a.w;
              }
            }
            float4* op = reinterpret_cast<float4*>(g.out + o0);
#pragma unroll
            for (int j = 0; j < 8; j++) op[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
          }
        }
        kcol += w;
      }
    }
    umma::fence_before_sync();
    __syncthreads();
  }
  if (s_abort && threadIdx.x == 0) set_err(p.err, 2);
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

// ---- backward: weight gradients -------------------------------------------------------

__host__ __device__ constexpr size_t bwd_weight_smem_bytes(int k_in) {
  return 1024 + static_cast<size_t>(kRows) * k_in * 2 /* A */ + kRows * kHid * 2 /* dz1 */ +
         kRows * kHid * 2 /* a1 */ + kRows * 128 * 2 /* dy */ + 256;
}

__host__ __device__ constexpr int part_stride(int k_in, int n_out) {
  return kHid * k_in + kHid + n_out * kHid + n_out;
}

__global__ void __launch_bounds__(kThreads, 1) k_mlp_bwd_weight(MlpBwdWeight p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = align1024(smem_raw);
  uint8_t* as = base;                         // [128][k_in] blocks of 64 cols (16 KB each)
  uint8_t* dzs = as + kRows * p.k_in * 2;     // [128][128]
  uint8_t* a1s = dzs + kRows * kHid * 2;      // [128][128]
  uint8_t* dys = a1s + kRows * kHid * 2;      // [128][n_out]
  uint64_t* bars = reinterpret_cast<uint64_t*>(dys + kRows * 128 * 2);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 1);
  __shared__ int s_abort;
  __shared__ float s_db[2][kHid];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    umma::mbar_init(&bars[0], 1);
    umma::mbar_fence_init();
    s_abort = 0;
  }
  if (warp == 0) umma::tmem_alloc(tmem_slot, 512);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t dw1 = tmem, dw2 = tmem + p.k_in;  // dW1 [128 hid][k_in], dW2^T [128 hid][n_out]
  const uint32_t aa = umma::smem_addr(as), dza = umma::smem_addr(dzs);
  const uint32_t a1a = umma::smem_addr(a1s), dya = umma::smem_addr(dys);
  const int nchunk = p.k_in >= 128 ? 128 : p.k_in;
  // dW1 = dz1^T A : A-operand dz1^T [M=128 hid, K=rows] MN-major; B = A^T [N=k_in chunk, K=rows] MN-major
  const uint32_t idesc_w1 = umma::idesc_bf16(kHid, nchunk, true, true);
  // dW2^T = a1^T dy : A-operand a1^T [M=128, K=rows] MN-major; B = dy^T [N=n_out, K=rows] MN-major
  const uint32_t idesc_w2 = umma::idesc_bf16(kHid, p.n_out, true, true);

  float db1 = 0.f, db2 = 0.f;  // thread t < 128: column t of dz1; t >= 128: column t-128 of dy
  const int ntiles = p.rows / kRows;
  uint32_t it = 0;
  bool any = false;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
    const int row0 = tile * kRows;
    if (it > 0) {
      if (!umma::mbar_wait(&bars[0], (it - 1) & 1)) s_abort = 1;
      __syncthreads();
      if (s_abort) break;
    }
    int kcol = 0;
    for (int s = 0; s < p.nseg; s++) {
      stage_segment(p.seg[s], row0, as + (kcol >> 6) * (kRows * 128));
      kcol += p.seg[s].width;
    }
    stage_matrix(p.dz1 + static_cast<size_t>(row0) * kHid, kRows, kHid, dzs);
    stage_matrix(p.a1 + static_cast<size_t>(row0) * kHid, kRows, kHid, a1s);
    stage_f32(p.dy, p.n_out, row0, dys);
    // bias gradients from global (fp32 dy, bf16 dz1), fixed row order
    if (threadIdx.x < kHid) {
      const int c = threadIdx.x;
      for (int rr = 0; rr < kRows; rr++) db1 += __bfloat162float(p.dz1[static_cast<size_t>(row0 + rr) * kHid + c]);
    } else if (threadIdx.x - kHid < p.n_out) {
      const int c = threadIdx.x - kHid;
      for (int rr = 0; rr < kRows; rr++) db2 += p.dy[static_cast<size_t>(row0 + rr) * p.n_out + c];
    }
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
      for (int k = 0; k < kRows; k += 16) {  // K = rows of the tile; 16 rows = 2 KB
        const uint64_t ad = umma::desc_mnmajor(dza + k * 128, kRows * 128);
        for (int n0 = 0; n0 < p.k_in; n0 += nchunk) {
          const uint64_t bd = umma::desc_mnmajor(aa + (n0 >> 6) * (kRows * 128) + k * 128, kRows * 128);
          umma::mma_bf16(dw1 + n0, ad, bd, idesc_w1, (it > 0 || k > 0) ? 1u : 0u);
        }
        const uint64_t a2 = umma::desc_mnmajor(a1a + k * 128, kRows * 128);
        const uint64_t b2 = umma::desc_mnmajor(dya + k * 128, kRows * 128);
        umma::mma_bf16(dw2, a2, b2, idesc_w2, (it > 0 || k > 0) ? 1u : 0u);
      }
      umma::commit(&bars[0]);
    }
    any = true;
  }
  if (any && !s_abort) {
    if (!umma::mbar_wait(&bars[0], (it - 1) & 1)) s_abort = 1;
  }
  __syncthreads();
  float* part = p.part + static_cast<size_t>(blockIdx.x) * part_stride(p.k_in, p.n_out);
  if (threadIdx.x < kHid) s_db[0][threadIdx.x] = db1;
  else if (threadIdx.x - kHid < p.n_out) s_db[1][threadIdx.x - kHid] = db2;
  __syncthreads();
  if (!s_abort) {
    umma::fence_after_sync();
    const int lane_base = (warp & 3) * 32;
    const int r = lane_base + lane;  // hidden unit
    const int half = warp >> 2;
    // dW1 [hid][k_in]
    const int per_half = p.k_in / 2;
    for (int cc = 0; cc < per_half; cc += 32) {
      const int col0 = half * per_half + cc;
      float v[32];
      if (any) umma::tmem_ld32(dw1 + (static_cast<uint32_t>(lane_base) << 16) + col0, v);
      else for (int j = 0; j < 32; j++) v[j] = 0.f;
      float4* op = reinterpret_cast<float4*>(part + static_cast<size_t>(r) * p.k_in + col0);
#pragma unroll
      for (int j = 0; j < 8; j++) op[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
    float* pw2 = part + kHid * p.k_in + kHid;  // dW2 [n_out][hid]
    const int per_half2 = p.n_out / 2;
    for (int cc = 0; cc < per_half2; cc += 32) {
      const int col0 = half * per_half2 + cc;
      float v[32];
      if (any) umma::tmem_ld32(dw2 + (static_cast<uint32_t>(lane_base) << 16) + col0, v);
      else for (int j = 0; j < 32; j++) v[j] = 0.f;
#pragma unroll
      for (int j = 0; j < 32; j++) pw2[static_cast<size_t>(col0 + j) * kHid + r] = v[j];
    }
    if (threadIdx.x < kHid) part[kHid * p.k_in + threadIdx.x] = s_db[0][threadIdx.x];
    if (threadIdx.x < p.n_out) pw2[p.n_out * kHid + threadIdx.x] = s_db[1][threadIdx.x];
  } else if (threadIdx.x == 0) {
    set_err(p.err, 3);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

// ---- small kernels -------------------------------------------------------------------

// grad[i] = sum over CTAs b (in order) of part[b][i]
__global__ void k_reduce_parts(const float* __restrict__ part, int nparts, int n, float* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int b = 0; b < nparts; b++) s += part[static_cast<size_t>(b) * n + i];
  grad[i] = s;
}

// de_tot[k][c] = de[k][c] + (nbr[k][c] >= 0 ? dagg[c] : 0)     (aggregation backward)
__global__ void k_agg_backward(const float* __restrict__ de, const float* __restrict__ dagg,
                               const int32_t* __restrict__ nbr, int Tp, float* __restrict__ out) {
  const size_t n = static_cast<size_t>(3) * Tp * kHid / 4;
  for (size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t e = q * 4 / kHid;  // edge row
    const int c = static_cast<int>(e % Tp);
    const int col = static_cast<int>((q * 4) % kHid);
    float4 a = de ? reinterpret_cast<const float4*>(de)[q] : make_float4(0.f, 0.f, 0.f, 0.f);
    if (nbr[e] >= 0) {
      const float4 g = *reinterpret_cast<const float4*>(dagg + static_cast<size_t>(c) * kHid + col);
      a.x += g.x; a.y += g.y; a.z += g.z; a.w += g.w;
    }
    reinterpret_cast<float4*>(out)[q] = a;
  }
}

// dh[c] = dh_in[c] + sum_k ddst[k][c] + sum_k dsrc[rev[k][c]]   (gather backward)
__global__ void k_node_backward(const float* __restrict__ dh_in, const float* __restrict__ ddst,
                                const float* __restrict__ dsrc, const int32_t* __restrict__ rev, int Tp,
                                float* __restrict__ out) {
  const size_t n = static_cast<size_t>(Tp) * kHid / 4;
  for (size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(q * 4 / kHid);
    const int col = static_cast<int>((q * 4) % kHid);
    float4 a = reinterpret_cast<const float4*>(dh_in)[q];
    for (int k = 0; k < 3; k++) {
      const float4 g = *reinterpret_cast<const float4*>(ddst + (static_cast<size_t>(k) * Tp + c) * kHid + col);
      a.x += g.x; a.y += g.y; a.z += g.z; a.w += g.w;
    }
    for (int k = 0; k < 3; k++) {
      const int e = rev[static_cast<size_t>(k) * Tp + c];
      if (e < 0) continue;
      const float4 g = *reinterpret_cast<const float4*>(dsrc + static_cast<size_t>(e) * kHid + col);
      a.x += g.x; a.y += g.y; a.z += g.z; a.w += g.w;
    }
    reinterpret_cast<float4*>(out)[q] = a;
  }
}

// Masked mean-squared error over the first `nout` columns of y (row stride ld):
// per-block partial loss and dy = 2 (y - t) w / norm.
__global__ void k_mse(const float* __restrict__ y, int ld, const float* __restrict__ target,
                      const float* __restrict__ wmask, int Tp, int nout, float norm, float* __restrict__ dy,
                      float* __restrict__ loss_part) {
  __shared__ float red[256];
  float acc = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Tp; i += gridDim.x * blockDim.x) {
    const float w = wmask[i];
    for (int j = 0; j < ld; j++) {
      float g = 0.f;
      if (j < nout) {
        const float d = y[static_cast<size_t>(i) * ld + j] - target[static_cast<size_t>(i) * nout + j];
        acc += w * d * d;
        g = 2.f * w * d / norm;
      }
      dy[static_cast<size_t>(i) * ld + j] = g;
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0] / norm;
}

// Adam on fp32 master weights; writes the bf16 copy the kernels read.
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, bf16* __restrict__ wb, int n, float lr, float b1,
                       float b2, float eps, float bc1, float bc2, float wd, float clip_scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] * clip_scale;
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i];
  wi -= lr * ((mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * wi);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
}

__global__ void k_sumsq(const float* __restrict__ g, int n, float* __restrict__ out_part) {
  __shared__ float red[256];
  float acc = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += g[i] * g[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out_part[blockIdx.x] = red[0];
}

}  // namespace gnn
}  // namespace storm

// ---- C-ABI launchers (include/storm_gnn.h) ------------------------------------------

#include <atomic>
#include <string>

#include "../../include/storm_gnn.h"

namespace storm {
int set_error(int code, const std::string& msg);
void clear_error();
}  // namespace storm

namespace {

using namespace storm::gnn;

std::atomic<int64_t> g_launches{0};
constexpr int kMinBwdSmem = 120 * 1024;  // one CTA per SM: the backward kernels take all of TMEM

int cuda_check(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return storm::set_error(STORM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return STORM_OK;
}

int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

bool valid_width(int w) { return w == 64 || w == 128; }

int check_shape(int rows, int nseg, int k_in, int n_out, const int* widths) {
  if (rows <= 0 || rows % kRows) return storm::set_error(STORM_ERR_ARG, "rows must be a positive multiple of 128");
  if (nseg < 1 || nseg > kMaxSeg) return storm::set_error(STORM_ERR_ARG, "1 to 3 input segments");
  int k = 0;
  for (int s = 0; s < nseg; s++) {
    if (!valid_width(widths[s])) return storm::set_error(STORM_ERR_ARG, "segment width must be 64 or 128");
    k += widths[s];
  }
  if (k != k_in || k_in > 384) return storm::set_error(STORM_ERR_ARG, "k_in must equal the segment widths (<= 384)");
  if (n_out != 64 && n_out != 128) return storm::set_error(STORM_ERR_ARG, "n_out must be 64 or 128");
  return STORM_OK;
}

Seg to_seg(const StormGnnSeg& s) {
  Seg o;
  o.src = static_cast<const bf16*>(s.src);
  o.idx = s.idx;
  o.width = s.width;
  o.agg = s.agg;
  o.agg_stride = s.agg_stride;
  o.nbr = s.nbr;
  return o;
}

int check_segs(const StormGnnSeg* seg, int nseg, int rows) {
  for (int s = 0; s < nseg; s++) {
    if (!seg[s].src) return storm::set_error(STORM_ERR_ARG, "segment source is NULL");
    if (seg[s].agg && (!seg[s].nbr || seg[s].agg_stride < rows))
      return storm::set_error(STORM_ERR_ARG, "aggregation segment needs nbr and agg_stride >= rows");
  }
  return STORM_OK;
}

int grid_for(int rows) {
  const int tiles = rows / kRows;
  return tiles < num_sms() ? tiles : num_sms();
}

}  // namespace

extern "C" {

int32_t storm_gnn_grad_size(int32_t k_in, int32_t n_out) { return part_stride(k_in, n_out); }

size_t storm_gnn_weight_scratch_bytes(int32_t k_in, int32_t n_out) {
  return static_cast<size_t>(num_sms()) * part_stride(k_in, n_out) * sizeof(float);
}

int storm_gnn_mlp_forward(const StormGnnMlpFwd* a, int32_t* dev_err, void* stream) {
  storm::clear_error();
  if (!a) return storm::set_error(STORM_ERR_ARG, "NULL arguments");
  int widths[kMaxSeg] = {0, 0, 0};
  for (int s = 0; s < a->nseg && s < kMaxSeg; s++) widths[s] = a->seg[s].width;
  int rc = check_shape(a->rows, a->nseg, a->k_in, a->n_out, widths);
  if (rc) return rc;
  if ((rc = check_segs(a->seg, a->nseg, a->rows))) return rc;
  if (!a->w1 || !a->b1 || !a->w2 || !a->b2 || !a->out) return storm::set_error(STORM_ERR_ARG, "NULL weight or output");
  MlpFwd p{};
  p.rows = a->rows; p.nseg = a->nseg; p.k_in = a->k_in; p.n_out = a->n_out;
  for (int s = 0; s < a->nseg; s++) p.seg[s] = to_seg(a->seg[s]);
  p.w1 = static_cast<const bf16*>(a->w1); p.b1 = a->b1;
  p.w2 = static_cast<const bf16*>(a->w2); p.b2 = a->b2;
  p.res = static_cast<const bf16*>(a->res); p.out = static_cast<bf16*>(a->out);
  p.out_f32 = a->out_f32; p.a1_save = static_cast<bf16*>(a->a1_save); p.err = dev_err;
  const size_t smem = fwd_smem_bytes(a->k_in, a->n_out);
  cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  k_mlp_fwd<<<grid_for(a->rows), kFwdThreads, smem, static_cast<cudaStream_t>(stream)>>>(p);
  g_launches++;
  return cuda_check("k_mlp_fwd");
}

int storm_gnn_mlp_backward_data(const StormGnnMlpBwdData* a, int32_t* dev_err, void* stream) {
  storm::clear_error();
  if (!a) return storm::set_error(STORM_ERR_ARG, "NULL arguments");
  int rc = check_shape(a->rows, a->nseg, a->k_in, a->n_out, a->seg_width);
  if (rc) return rc;
  if (!a->dy || !a->a1 || !a->w1 || !a->w2) return storm::set_error(STORM_ERR_ARG, "NULL input");
  MlpBwdData p{};
  p.rows = a->rows; p.nseg = a->nseg; p.k_in = a->k_in; p.n_out = a->n_out;
  for (int s = 0; s < a->nseg; s++) {
    p.seg_width[s] = a->seg_width[s];
    p.dseg[s].out = a->dseg[s];
    p.dseg[s].add = a->dseg_add[s];
  }
  p.dy = a->dy; p.a1 = static_cast<const bf16*>(a->a1);
  p.w1 = static_cast<const bf16*>(a->w1); p.w2 = static_cast<const bf16*>(a->w2);
  p.dz1_save = static_cast<bf16*>(a->dz1_save); p.err = dev_err;
  size_t smem = bwd_data_smem_bytes(a->k_in, a->n_out);
  if (smem < static_cast<size_t>(kMinBwdSmem)) smem = kMinBwdSmem;
  cudaFuncSetAttribute(k_mlp_bwd_data, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  k_mlp_bwd_data<<<grid_for(a->rows), kThreads, smem, static_cast<cudaStream_t>(stream)>>>(p);
  g_launches++;
  return cuda_check("k_mlp_bwd_data");
}

int storm_gnn_mlp_backward_weight(const StormGnnMlpBwdWeight* a, float* grad, void* scratch, size_t scratch_bytes,
                                  int32_t* dev_err, void* stream) {
  storm::clear_error();
  if (!a || !grad || !scratch) return storm::set_error(STORM_ERR_ARG, "NULL arguments");
  int widths[kMaxSeg] = {0, 0, 0};
  for (int s = 0; s < a->nseg && s < kMaxSeg; s++) widths[s] = a->seg[s].width;
  int rc = check_shape(a->rows, a->nseg, a->k_in, a->n_out, widths);
  if (rc) return rc;
  if ((rc = check_segs(a->seg, a->nseg, a->rows))) return rc;
  if (!a->dy || !a->a1 || !a->dz1) return storm::set_error(STORM_ERR_ARG, "NULL input");
  const int grid = grid_for(a->rows);
  const int n = part_stride(a->k_in, a->n_out);
  if (scratch_bytes < static_cast<size_t>(grid) * n * sizeof(float))
    return storm::set_error(STORM_ERR_ARG, "weight-gradient scratch too small");
  MlpBwdWeight p{};
  p.rows = a->rows; p.nseg = a->nseg; p.k_in = a->k_in; p.n_out = a->n_out;
  for (int s = 0; s < a->nseg; s++) p.seg[s] = to_seg(a->seg[s]);
  p.dy = a->dy; p.a1 = static_cast<const bf16*>(a->a1); p.dz1 = static_cast<const bf16*>(a->dz1);
  p.part = static_cast<float*>(scratch); p.err = dev_err;
  size_t smem = bwd_weight_smem_bytes(a->k_in);
  if (smem < static_cast<size_t>(kMinBwdSmem)) smem = kMinBwdSmem;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaFuncSetAttribute(k_mlp_bwd_weight, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  k_mlp_bwd_weight<<<grid, kThreads, smem, st>>>(p);
  k_reduce_parts<<<(n + 255) / 256, 256, 0, st>>>(p.part, grid, n, grad);
  g_launches += 2;
  return cuda_check("k_mlp_bwd_weight");
}

int storm_gnn_agg_backward(const float* de, const float* dagg, const int32_t* nbr, int32_t Tp, float* out,
                           void* stream) {
  storm::clear_error();
  if (!dagg || !nbr || !out || Tp <= 0 || Tp % kRows) return storm::set_error(STORM_ERR_ARG, "bad arguments");
  k_agg_backward<<<num_sms() * 4, 256, 0, static_cast<cudaStream_t>(stream)>>>(de, dagg, nbr, Tp, out);
  g_launches++;
  return cuda_check("k_agg_backward");
}

int storm_gnn_node_backward(const float* dh, const float* ddst, const float* dsrc, const int32_t* rev, int32_t Tp,
                            float* out, void* stream) {
  storm::clear_error();
  if (!dh || !ddst || !dsrc || !rev || !out || Tp <= 0 || Tp % kRows)
    return storm::set_error(STORM_ERR_ARG, "bad arguments");
  k_node_backward<<<num_sms() * 4, 256, 0, static_cast<cudaStream_t>(stream)>>>(dh, ddst, dsrc, rev, Tp, out);
  g_launches++;
  return cuda_check("k_node_backward");
}

int storm_gnn_mse(const float* y, int32_t ld, const float* target, const float* w, int32_t Tp, int32_t nout,
                  float norm, float* dy, float* loss_part, void* stream) {
  storm::clear_error();
  if (!y || !target || !w || !dy || !loss_part || Tp <= 0 || nout <= 0 || nout > ld || !(norm > 0.f))
    return storm::set_error(STORM_ERR_ARG, "bad arguments");
  k_mse<<<148, 256, 0, static_cast<cudaStream_t>(stream)>>>(y, ld, target, w, Tp, nout, norm, dy, loss_part);
  g_launches++;
  return cuda_check("k_mse");
}

int storm_gnn_adam(float* w, float* m, float* v, const float* g, void* w_bf16, int32_t n, float lr, float beta1,
                   float beta2, float eps, int32_t step, float weight_decay, float grad_scale, void* stream) {
  storm::clear_error();
  if (!w || !m || !v || !g || n <= 0 || step < 1) return storm::set_error(STORM_ERR_ARG, "bad arguments");
  const float bc1 = 1.f - powf(beta1, static_cast<float>(step));
  const float bc2 = 1.f - powf(beta2, static_cast<float>(step));
  k_adam<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      w, m, v, g, static_cast<bf16*>(w_bf16), n, lr, beta1, beta2, eps, bc1, bc2, weight_decay, grad_scale);
  g_launches++;
  return cuda_check("k_adam");
}

int storm_gnn_sumsq(const float* g, int32_t n, float* out_part, void* stream) {
  storm::clear_error();
  if (!g || !out_part || n <= 0) return storm::set_error(STORM_ERR_ARG, "bad arguments");
  k_sumsq<<<148, 256, 0, static_cast<cudaStream_t>(stream)>>>(g, n, out_part);
  g_launches++;
  return cuda_check("k_sumsq");
}

int64_t storm_gnn_kernel_launches(void) { return g_launches.load(); }

}  // extern "C"
