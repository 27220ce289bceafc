/*
 * storm_gnn.h -- C-ABI of the warm-start network kernels (sm_100a).
 *
 * No counterpart in the reference: SToRM starts a steady run from the initial
 * condition the user supplies (read_data / initial-condition input), and the
 * solverFVT loop (Source_xsy-64bit/solverFVT.f90:129-478) iterates from there.  These
 * entry points run a message-passing network on the cell-dual graph that predicts
 * an initial h, hu, hv; the caller hands the prediction to storm_fvt_set_state (or
 * storm_fvt_set_scenario_state) and the solver runs on to its own stop test.
 *
 * All pointers are device pointers (bf16 = 16-bit bfloat, fp32 = float) and every
 * launch goes on the given CUDA stream (NULL: the legacy default stream).  Row counts
 * are multiples of 128.  Matrices are row-major.  Return values follow storm_fvt.h
 * (0 or a negative STORM_ERR_* code; message from storm_fvt_last_error()).
 *
 * Graph layout: cells padded to Tp (a multiple of 128); the three directed edge rows
 * of cell c are k*Tp + c (k = 0, 1, 2, its local faces), carrying the message from
 * neighbour nbr[k*Tp + c] (or -1: no neighbour) into c.
 */
#ifndef STORM_GNN_H
#define STORM_GNN_H

#include <stddef.h>
#include <stdint.h>

#include "storm_fvt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One 64- or 128-wide segment of an MLP input row. */
typedef struct StormGnnSeg {
  const void* src;       /* bf16 [*][width]                                         */
  const int32_t* idx;    /* row map (NULL: identity); a negative entry reads zeros  */
  int32_t width;         /* 64 or 128                                                */
  int32_t agg;           /* 1: row r is the sum of src rows r + k*agg_stride, k<3,
                            whose nbr entry is >= 0 (message aggregation)           */
  int32_t agg_stride;
  const int32_t* nbr;    /* [3*agg_stride] (agg only)                                */
} StormGnnSeg;

/* out = res + W2 relu(W1 [seg0 | seg1 | seg2] + b1) + b2  (rows x n_out) */
typedef struct StormGnnMlpFwd {
  int32_t rows, nseg, k_in, n_out; /* k_in = sum of segment widths; n_out 64 or 128 */
  StormGnnSeg seg[3];
  const void* w1;       /* bf16 [128][k_in] */
  const float* b1;      /* [128]            */
  const void* w2;       /* bf16 [n_out][128] */
  const float* b2;      /* [n_out]          */
  const void* res;      /* bf16 [rows][n_out] or NULL */
  void* out;            /* bf16 [rows][n_out] */
  float* out_f32;       /* optional fp32 copy [rows][n_out] */
  void* a1_save;        /* optional bf16 [rows][128] hidden activation (training) */
} StormGnnMlpFwd;

/* Data gradients: dz1 = (dy W2) * (a1 > 0); dseg[s] = add[s] + (dz1 W1)[:, segment s] */
typedef struct StormGnnMlpBwdData {
  int32_t rows, nseg, k_in, n_out;
  int32_t seg_width[3];
  float* dseg[3];        /* fp32 [rows][width] or NULL (not needed) */
  const float* dseg_add[3]; /* fp32 addend or NULL */
  const float* dy;       /* fp32 [rows][n_out] */
  const void* a1;        /* bf16 [rows][128]   */
  const void* w1;        /* bf16 [128][k_in]   */
  const void* w2;        /* bf16 [n_out][128]  */
  void* dz1_save;        /* bf16 [rows][128]   */
} StormGnnMlpBwdData;

/* Weight gradients: grad = [dW1 (128 x k_in) | db1 (128) | dW2 (n_out x 128) | db2 (n_out)] */
typedef struct StormGnnMlpBwdWeight {
  int32_t rows, nseg, k_in, n_out;
  StormGnnSeg seg[3];
  const float* dy;       /* fp32 [rows][n_out] */
  const void* a1;        /* bf16 [rows][128]   */
  const void* dz1;       /* bf16 [rows][128]   */
} StormGnnMlpBwdWeight;

/* Number of floats of one gradient vector (and of one per-CTA partial). */
STORM_FVT_API int32_t storm_gnn_grad_size(int32_t k_in, int32_t n_out);
/* Bytes of device scratch storm_gnn_mlp_backward_weight needs. */
STORM_FVT_API size_t storm_gnn_weight_scratch_bytes(int32_t k_in, int32_t n_out);

STORM_FVT_API int storm_gnn_mlp_forward(const StormGnnMlpFwd* a, int32_t* dev_err, void* stream);
STORM_FVT_API int storm_gnn_mlp_backward_data(const StormGnnMlpBwdData* a, int32_t* dev_err, void* stream);
/* grad (fp32, storm_gnn_grad_size floats) is overwritten; scratch as sized above. */
STORM_FVT_API int storm_gnn_mlp_backward_weight(const StormGnnMlpBwdWeight* a, float* grad, void* scratch,
                                                size_t scratch_bytes, int32_t* dev_err, void* stream);

/* out[k*Tp+c] = de[k*Tp+c] (or 0 when de is NULL) + (nbr[k*Tp+c] >= 0 ? dagg[c] : 0), 128 wide */
STORM_FVT_API int storm_gnn_agg_backward(const float* de, const float* dagg, const int32_t* nbr, int32_t Tp,
                                         float* out, void* stream);
/* out[c] = dh[c] + sum_k ddst[k*Tp+c] + sum_k dsrc[rev[k*Tp+c]] (rev < 0 skipped), 128 wide */
STORM_FVT_API int storm_gnn_node_backward(const float* dh, const float* ddst, const float* dsrc,
                                          const int32_t* rev, int32_t Tp, float* out, void* stream);
/* loss_part[b] (b < 148) = per-block sum of w (y - t)^2 / norm over the first nout of ld columns;
   dy = 2 w (y - t) / norm (zero in the other columns). */
STORM_FVT_API int storm_gnn_mse(const float* y, int32_t ld, const float* target, const float* w, int32_t Tp,
                                int32_t nout, float norm, float* dy, float* loss_part, void* stream);
/* Adam step on fp32 master weights (with decoupled weight decay), writing the bf16 copy. */
STORM_FVT_API int storm_gnn_adam(float* w, float* m, float* v, const float* g, void* w_bf16, int32_t n, float lr,
                                 float beta1, float beta2, float eps, int32_t step, float weight_decay,
                                 float grad_scale, void* stream);
/* out_part[b] (b < 148) = per-block sum of g^2 */
STORM_FVT_API int storm_gnn_sumsq(const float* g, int32_t n, float* out_part, void* stream);
/* Kernels launched through this header since library load. */
STORM_FVT_API int64_t storm_gnn_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* STORM_GNN_H */
