// api.cu -- the C-ABI entry points of include/storm_fvt.h (handle, state, stepping).
//
// storm_fvt_create copies the prepared mesh to HBM in the reordered SoA layout and
// captures one full iteration (all RK stages, friction, reductions) as a CUDA graph;
// storm_fvt_step replays the graph `nsteps` times on the handle's stream, polling
// the device-side stop flag every few iterations in steady mode, so the host never
// synchronises inside an iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "fvt_device.cuh"
#include "storm_internal.h"

namespace storm {

__global__ void k_init(Dev d, int c0);
__global__ void k_init_final(Dev d, int sid);
__global__ void k_final(Dev d);

static thread_local std::string g_err;

int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
void clear_error() { g_err.clear(); }

}  // namespace storm

using namespace storm;

struct StormFvtHandle {
  StormFvtOptions opt{};
  std::vector<HostLayout> parts;  // per-scenario layouts (permutations for state I/O)
  std::vector<ScenarioInfo> info; // placement of each scenario in the merged arrays
  HostLayout L;                   // merged layout that is on the device
  int nscen = 1;
  std::vector<uint8_t> have_scen_state;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;       // boundary kernel, overlapped with k_flux
  cudaEvent_t fork_ev[4] = {}, join_ev[4] = {}, eflux_ev[4] = {};
  void* arena = nullptr;
  void* arena32 = nullptr;  // FP32 geometry copies (mixed precision only)
  Dev d{};
  Geo<double> gd{};  // FP64 views
  Geo<float> gf{};   // FP32 copies (mixed precision)
  bool mixed = false;
  Scalars* sc_host = nullptr;  // pinned, [nscen]
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int kernels_per_step = 0;
  int64_t launches = 0;
  size_t bc_smem = 0;
  bool have_state = false;
  bool timing = false;
  double last_step_ms = 0.0, last_flux_ms = 0.0;
  int64_t last_flux_launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> fev;  // event pairs of the timing mode
  std::vector<int> fev_class;    // kernel class of each pair
  double kt_ms[8] = {0};         // per-class totals of the last timed call
  int64_t kt_n[8] = {0};
  // block sizes of the stage kernels (storm_fvt_autotune picks them)
  // block sizes of the node, gradient, edge-flux and cell kernels: the autotuner's
  // choice on the 2M meander (FP64; the mixed path takes 128 for the edge fluxes)
  int bs_node = 128, bs_grad = 64, bs_eflux = 64, bs_flux = 64;
  // output pass (storm_fvt_output_vertices): device buffers, allocated at first use
  void* out_buf = nullptr;
  size_t out_bytes = 0;
  void* halo_buf = nullptr;  // linked partitions: halo slots, owner slots, halo mask
  double* io_host = nullptr;  // pinned staging of state transfers (grown on demand)
  size_t io_n = 0;
  // fused stage kernel: tile plan, its device copy, the second velocity buffer
  TilePlan tiles;
  TileDev td{};
  void* tile_buf = nullptr;
  size_t tile_smem = 0;
  int tile_grid = 0;        // persistent grid of k_tile: resident CTAs on all SMs
  bool tiles_ok = false;    // plan built and within the shared-memory limit
  bool want_tiles = false;  // storm_fvt_set_stage_path / storm_fvt_autotune (phase kernels by default)
  bool use_tiles = false;   // the captured iteration runs k_tile
  bool fuse_nodes = true;   // k_tile computes the vertex depths (else k_node runs before it)
  int32_t* bc_nodes = nullptr;  // vertices of the boundary cells (device, in tile_buf)
  int n_bc_nodes = 0;
  // one part of a mesh per process: the cells this part sends / receives (device slots)
  void* xchg_buf = nullptr;
  int32_t *send_slots = nullptr, *recv_slots = nullptr;
  int n_send = 0, n_recv = 0;
  double *u_a2 = nullptr, *v_a2 = nullptr;
};

namespace {

constexpr int kFluxThreads = 128;
constexpr int kRed = 256;
constexpr int kFinalThreadsHost = 512;  // k_final's block (kFinalThreads in fvt_kernels.cu)

#define CK(call)                                                                                     \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return set_error(STORM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
  } while (0)

int check_options(const StormFvtOptions& o) {
  if (o.rkorder < 1 || o.rkorder > 3) return set_error(STORM_ERR_ARG, "Incorrect Runge-Kutta order (1, 2 or 3)");
  if (o.opt_limiter < 0 || o.opt_limiter > 2) return set_error(STORM_ERR_ARG, "opt_limiter must be 0, 1 or 2");
  if (o.btype != 0 && o.btype != 1) return set_error(STORM_ERR_ARG, "btype must be 0 or 1");
  if (o.opt_friction < 0 || o.opt_friction > 4)
    return set_error(STORM_ERR_UNSUPPORTED, "opt_friction must be 0..4 (5, the vegetation model, is not built)");
  if (o.flux < 0 || o.flux > 2) return set_error(STORM_ERR_ARG, "flux must be ROE, HLL or RUSANOV");
  if (o.stop_cr != 0 && o.stop_cr != 1) return set_error(STORM_ERR_ARG, "stop_cr must be 0 or 1");
  if (o.precision != STORM_PREC_FP64 && o.precision != STORM_PREC_MIXED)
    return set_error(STORM_ERR_ARG, "precision must be STORM_PREC_FP64 or STORM_PREC_MIXED");
  if (!(o.h_dry > 0.0) || !(o.h_wet >= o.h_dry)) return set_error(STORM_ERR_ARG, "need 0 < h_dry <= h_wet");
  if (!(o.cfl > 0.0)) return set_error(STORM_ERR_ARG, "cfl must be positive");
  if (o.rsavg_passes < 0 || o.rsavg_passes > 64) return set_error(STORM_ERR_ARG, "rsavg_passes must be 0..64");
  if (o.rsavg_passes > 0 && !(o.rsavg_eps > 0.0 && o.rsavg_eps <= 1.0))
    return set_error(STORM_ERR_ARG, "rsavg_eps must be in (0, 1]");
  if (o.rsavg_passes > 0 && o.rsavg_order != 1)
    return set_error(STORM_ERR_UNSUPPORTED,
                     "residual smoothing in cell index order is serial; the GPU runs rsavg_order 1 (by colour)");
  for (int i = 0; i < 2; i++)
    if (o.reserved[i]) return set_error(STORM_ERR_ARG, "reserved option fields must be zero");
  return 0;
}

// Device arena: every buffer 256-byte aligned inside one allocation.
struct Arena {
  size_t off = 0;
  std::vector<std::pair<size_t, size_t>> items;
  size_t take(size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  }
};

template <class T>
T* at(void* base, size_t off) {
  return reinterpret_cast<T*>(static_cast<char*>(base) + off);
}

// Kernel classes of the per-kernel timing mode.
enum { KT_NODE = 0, KT_GRAD, KT_BC, KT_FLUX, KT_FRIC, KT_FINAL, KT_EFLUX, KT_TILE, KT_COUNT };
static_assert(KT_COUNT <= 8, "per-class timing arrays hold 8 classes");

constexpr int kTileCellsHost = 256;   // cell slots per tile of k_tile
constexpr int kTileThreadsHost = 256;

// One iteration (only = -1), or only its RK stage `only` (1..K), or only its friction
// step and reductions (only = 0: the iteration cut of storm_fvt_iter_*).
int enqueue_step(StormFvtHandle* h, bool timing, size_t* fev_used, int only = -1) {
  const Dev& d = h->d;
  const int T = d.T, K = d.K;
  const int gT = (T + h->bs_grad - 1) / h->bs_grad;
  const int gF = (T + h->bs_flux - 1) / h->bs_flux;
  const int gE = (d.ne + h->bs_eflux - 1) / h->bs_eflux;
  // in timing mode every launch is bracketed by an event pair tagged with its class
  auto mark = [&](int cls) -> int {
    if (!timing) return 0;
    CK(cudaEventRecord(h->fev[*fev_used], h->stream));
    h->fev_class[*fev_used / 2] = cls;
    (*fev_used)++;
    return 0;
  };
  auto done = [&]() -> int {
    if (!timing) return 0;
    CK(cudaEventRecord(h->fev[(*fev_used)++], h->stream));
    return 0;
  };
  const bool linked = d.linked != 0;
  const bool rs = h->opt.rsavg_passes > 0;
  // the fused tile kernel where its plan exists; the phase kernels for culverts,
  // residual smoothing and linked partitions
  const bool fused = h->tiles_ok && h->want_tiles && !linked && d.ncv == 0 && !rs;
  h->use_tiles = fused;
  const double *u_in = d.u_a, *v_in = d.v_a;
  double *u_out = d.u_a, *v_out = d.v_a;
  auto launch = [&](int which, int grid, int block, size_t smem, cudaStream_t st, int s, const double* hs,
                    uint8_t* dry, uint8_t* dry_next) {
    StageLaunch L;
    L.which = which;
    L.grid = dim3(grid);
    L.block = dim3(block);
    L.smem = smem;
    L.stream = st;
    L.s = s;
    L.hs = hs;
    L.dry = dry;
    L.dry_next = dry_next;
    L.rku_prev = d.rku + (size_t)(s - 1) * T;
    L.rkv_prev = d.rkv + (size_t)(s - 1) * T;
    L.u_in = u_in;
    L.v_in = v_in;
    L.u_out = u_out;
    L.v_out = v_out;
    L.tiles = &h->td;
    launch_stage(L, d, h->gd, h->gf, h->mixed);
  };
  if (only < 0 && linked && !d.steady && d.dt_op != 0) launch_link_dt(d, h->stream);
  for (int s = 1; s <= K; s++) {
    const double* hs = d.rkh + (size_t)(s - 1) * T;
    uint8_t* dry = (s & 1) ? d.dry_a : d.dry_b;
    uint8_t* dry_next = (s & 1) ? d.dry_b : d.dry_a;
    const int gB = (d.nbc_cells + kFluxThreads - 1) / kFluxThreads;
    if (fused) {  // stage s reads one velocity buffer and writes the other
      u_in = (s & 1) ? d.u_a : h->u_a2;
      v_in = (s & 1) ? d.v_a : h->v_a2;
      u_out = (s & 1) ? h->u_a2 : d.u_a;
      v_out = (s & 1) ? h->v_a2 : d.v_a;
    }
    if (only >= 0 && s != only) continue;
    const bool tile_nodes = fused && h->td.nodes;
    if (!tile_nodes) {
      if (mark(KT_NODE)) return STORM_ERR_CUDA;
      launch_node(d, hs, dry, nullptr, 0, h->bs_node, h->stream);
      if (done()) return STORM_ERR_CUDA;
    }
    if (fused) {
      const int nt = h->tile_grid;
      if (gB > 0 && !timing) {
        // the boundary cells' vertex depths (when the tiles compute the others), their
        // gradients and k_bc on the side stream beside k_tile; k_flux_bc updates those
        // cells once both are done
        CK(cudaEventRecord(h->fork_ev[s], h->stream));
        CK(cudaStreamWaitEvent(h->side, h->fork_ev[s], 0));
        if (tile_nodes) launch_node(d, hs, dry, h->bc_nodes, h->n_bc_nodes, 128, h->side);
        launch(STAGE_GRAD_BC, gB, kFluxThreads, 0, h->side, s, hs, dry, dry_next);
        if (d.nbdr > 0) launch(STAGE_BC, d.nbdr, 128, h->bc_smem, h->side, s, hs, dry, dry_next);
        CK(cudaEventRecord(h->join_ev[s], h->side));
        launch(STAGE_TILE, nt, kTileThreadsHost, h->tile_smem, h->stream, s, hs, dry, dry_next);
        CK(cudaStreamWaitEvent(h->stream, h->join_ev[s], 0));
        launch(STAGE_FLUX_BC, gB, kFluxThreads, 0, h->stream, s, hs, dry, dry_next);
      } else {
        if (gB > 0) {
          if (tile_nodes) {
            if (mark(KT_NODE)) return STORM_ERR_CUDA;
            launch_node(d, hs, dry, h->bc_nodes, h->n_bc_nodes, 128, h->stream);
            if (done()) return STORM_ERR_CUDA;
          }
          if (mark(KT_GRAD)) return STORM_ERR_CUDA;
          launch(STAGE_GRAD_BC, gB, kFluxThreads, 0, h->stream, s, hs, dry, dry_next);
          if (done()) return STORM_ERR_CUDA;
          if (d.nbdr > 0) {
            if (mark(KT_BC)) return STORM_ERR_CUDA;
            launch(STAGE_BC, d.nbdr, 128, h->bc_smem, h->stream, s, hs, dry, dry_next);
            if (done()) return STORM_ERR_CUDA;
          }
        }
        if (mark(KT_TILE)) return STORM_ERR_CUDA;
        launch(STAGE_TILE, nt, kTileThreadsHost, h->tile_smem, h->stream, s, hs, dry, dry_next);
        if (done()) return STORM_ERR_CUDA;
        if (gB > 0) {
          if (mark(KT_FLUX)) return STORM_ERR_CUDA;
          launch(STAGE_FLUX_BC, gB, kFluxThreads, 0, h->stream, s, hs, dry, dry_next);
          if (done()) return STORM_ERR_CUDA;
        }
      }
      continue;
    }
    if (mark(KT_GRAD)) return STORM_ERR_CUDA;
    launch(STAGE_GRAD, gT, h->bs_grad, 0, h->stream, s, hs, dry, dry_next);
    if (d.ncv > 0) launch(STAGE_CULVERT, (d.ncv + 127) / 128, 128, 0, h->stream, s, hs, dry, dry_next);
    if (done()) return STORM_ERR_CUDA;
    const int sF = rs ? STAGE_PHI : STAGE_FLUX, sFB = rs ? STAGE_PHI_BC : STAGE_FLUX_BC;
    if (d.nbdr > 0 && !timing) {
      // k_bc on the side stream overlaps k_eflux; the cells with an open-boundary face
      // (k_flux_bc: their own values, the edge fluxes and k_bc's contributions) are
      // then finished on the side stream beside k_flux of all the other cells
      CK(cudaEventRecord(h->fork_ev[s], h->stream));
      CK(cudaStreamWaitEvent(h->side, h->fork_ev[s], 0));
      launch(STAGE_BC, d.nbdr, 128, h->bc_smem, h->side, s, hs, dry, dry_next);
      if (gE > 0) launch(STAGE_EFLUX, gE, h->bs_eflux, 0, h->stream, s, hs, dry, dry_next);
      CK(cudaEventRecord(h->eflux_ev[s], h->stream));
      CK(cudaStreamWaitEvent(h->side, h->eflux_ev[s], 0));
      if (gB > 0) launch(sFB, gB, kFluxThreads, 0, h->side, s, hs, dry, dry_next);
      CK(cudaEventRecord(h->join_ev[s], h->side));
      launch(sF, gF, h->bs_flux, 0, h->stream, s, hs, dry, dry_next);
      CK(cudaStreamWaitEvent(h->stream, h->join_ev[s], 0));
    } else {
      if (d.nbdr > 0) {
        if (mark(KT_BC)) return STORM_ERR_CUDA;
        launch(STAGE_BC, d.nbdr, 128, h->bc_smem, h->stream, s, hs, dry, dry_next);
        if (done()) return STORM_ERR_CUDA;
      }
      if (gE > 0) {
        if (mark(KT_EFLUX)) return STORM_ERR_CUDA;
        launch(STAGE_EFLUX, gE, h->bs_eflux, 0, h->stream, s, hs, dry, dry_next);
        if (done()) return STORM_ERR_CUDA;
      }
      if (mark(KT_FLUX)) return STORM_ERR_CUDA;
      launch(sF, gF, h->bs_flux, 0, h->stream, s, hs, dry, dry_next);
      if (gB > 0) launch(sFB, gB, kFluxThreads, 0, h->stream, s, hs, dry, dry_next);
      if (done()) return STORM_ERR_CUDA;
    }
    if (rs) {  // solverFVT.f90:238-256, then the update of every cell
      if (mark(KT_FLUX)) return STORM_ERR_CUDA;
      const HostLayout& Lm = h->L;
      for (int k = 0; k < h->opt.rsavg_passes; k++)
        for (size_t c = 0; c + 1 < Lm.rs_off.size(); c++)
          launch_rsavg(d, Lm.rs_off[c], Lm.rs_off[c + 1] - Lm.rs_off[c], h->stream);
      launch(STAGE_UPDATE, (T + 127) / 128, 128, 0, h->stream, s, hs, dry, dry_next);
      if (done()) return STORM_ERR_CUDA;
    }
    // halo cells of linked partitions take their owners' new level and flags
    if (linked && d.nhalo > 0 && s < K) launch_halo(d, s, dry_next, nullptr, h->stream);
  }
  if (only > 0) {
    CK(cudaGetLastError());
    return 0;
  }
  if (linked && d.steady) launch_link_fric(d, h->stream);
  if (mark(KT_FRIC)) return STORM_ERR_CUDA;
  launch_fric(d, u_out, v_out, h->stream);
  if (done()) return STORM_ERR_CUDA;
  if (linked && d.nhalo > 0) launch_halo(d, 0, d.dry_a, d.dry_out, h->stream);
  if (mark(KT_FINAL)) return STORM_ERR_CUDA;
  k_final<<<d.nscen, kFinalThreadsHost, 0, h->stream>>>(d);
  if (done()) return STORM_ERR_CUDA;
  if (linked) launch_link(d, h->stream);
  CK(cudaGetLastError());
  return 0;
}

int capture_graph(StormFvtHandle* h) {
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  size_t dummy = 0;
  int rc = enqueue_step(h, false, &dummy);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return set_error(STORM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  h->graph = g;
  size_t n = 0;
  CK(cudaGraphGetNodes(g, nullptr, &n));
  h->kernels_per_step = (int)n;
  CK(cudaGraphInstantiate(&h->exec, g, 0));
  return 0;
}

void release(StormFvtHandle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  for (cudaEvent_t e : h->fev) cudaEventDestroy(e);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (int i = 0; i < 4; i++) {
    if (h->fork_ev[i]) cudaEventDestroy(h->fork_ev[i]);
    if (h->join_ev[i]) cudaEventDestroy(h->join_ev[i]);
    if (h->eflux_ev[i]) cudaEventDestroy(h->eflux_ev[i]);
  }
  if (h->side) cudaStreamDestroy(h->side);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (h->arena) cudaFree(h->arena);
  if (h->arena32) cudaFree(h->arena32);
  if (h->sc_host) cudaFreeHost(h->sc_host);
  if (h->out_buf) cudaFree(h->out_buf);
  if (h->halo_buf) cudaFree(h->halo_buf);
  if (h->tile_buf) cudaFree(h->tile_buf);
  if (h->xchg_buf) cudaFree(h->xchg_buf);
  if (h->io_host) cudaFreeHost(h->io_host);
  delete h;
}

// Shared memory and persistent grid of k_tile for the chosen variant (vertex depths in
// the tile or by k_node).
int configure_tiles(StormFvtHandle* h) {
  TileDev& t = h->td;
  t.nodes = h->fuse_nodes ? 1 : 0;
  const size_t smem = tile_smem_bytes(t, h->mixed);
  h->tile_smem = smem;
  if (smem > 48 * 1024) set_tile_smem_limit((int)smem);
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
  const int per_sm = std::max(1, tile_blocks_per_sm(h->mixed, smem));
  h->tile_grid = std::max(1, std::min(t.ntiles, nsm * per_sm));
  CK(cudaGetLastError());
  return 0;
}

// The tile plan of the fused stage kernel and its device copy.  A mesh whose tiles do
// not fit (more than 65,534 local cells or edges, or more shared memory than a block
// may have) keeps the phase kernels.
int upload_tiles(StormFvtHandle* h) {
  h->tiles_ok = false;
  TilePlan& P = h->tiles;
  if (build_tiles(h->L, kTileCellsHost, P) != 0 || check_tiles(h->L, P) != 0) {
    P = TilePlan();
    return 0;
  }
  TileDev& t = h->td;
  t.tc = P.tc; t.ntiles = P.ntiles; t.kst = P.kst;
  t.ns_max = P.ns_max; t.ng_max = P.ng_max; t.ne_max = P.ne_max; t.nn_max = P.nn_max;
  t.nodes = 1;
  const size_t smem = tile_smem_bytes(t, h->mixed);
  int dev_max = 0;
  CK(cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
  if (smem > (size_t)dev_max) {
    P = TilePlan();
    return 0;
  }
  Arena A;
  struct Up {
    size_t off;
    const void* src;
    size_t bytes;
  };
  std::vector<Up> ups;
  auto cpy = [&](const auto& vec) {
    using V = typename std::decay<decltype(vec)>::type::value_type;
    size_t o = A.take(sizeof(V) * std::max<size_t>(vec.size(), 1));
    if (!vec.empty()) ups.push_back({o, vec.data(), sizeof(V) * vec.size()});
    return o;
  };
  const size_t o_info = cpy(P.info), o_halo = cpy(P.halo), o_h1t3 = cpy(P.h1_t3), o_h1st = cpy(P.h1_st);
  const size_t o_lt3 = cpy(P.lt3), o_lst = cpy(P.lst), o_lfe = cpy(P.lfe), o_eloc = cpy(P.eloc);
  const size_t o_be = cpy(P.be), o_beloc = cpy(P.beloc);
  const size_t o_tn = cpy(P.tnode), o_tns = cpy(P.tn_start), o_tno = cpy(P.tn_own), o_tnc = cpy(P.tn_cells);
  const size_t o_lvt = cpy(P.lvt), o_h1vt = cpy(P.h1_vt), o_lw = cpy(P.lwall), o_bcn = cpy(P.bc_nodes);
  cudaError_t e = cudaMalloc(&h->tile_buf, A.off);
  if (e != cudaSuccess)
    return set_error(e == cudaErrorMemoryAllocation ? STORM_ERR_NOMEM : STORM_ERR_CUDA,
                     std::string("device allocation of the tile plan: ") + cudaGetErrorString(e));
  for (const Up& u : ups) CK(cudaMemcpy(static_cast<char*>(h->tile_buf) + u.off, u.src, u.bytes, cudaMemcpyHostToDevice));
  void* B = h->tile_buf;
  t.info = at<int32_t>(B, o_info); t.halo = at<int32_t>(B, o_halo);
  t.h1_t3 = at<uint16_t>(B, o_h1t3); t.h1_st = at<uint16_t>(B, o_h1st);
  t.lt3 = at<uint16_t>(B, o_lt3); t.lst = at<uint16_t>(B, o_lst); t.lfe = at<uint16_t>(B, o_lfe);
  t.eloc = at<uint32_t>(B, o_eloc); t.be = at<int32_t>(B, o_be); t.beloc = at<uint32_t>(B, o_beloc);
  t.tnode = at<int32_t>(B, o_tn); t.tn_start = at<int32_t>(B, o_tns); t.tn_own = at<uint8_t>(B, o_tno);
  t.tn_cells = at<uint16_t>(B, o_tnc); t.lvt = at<uint16_t>(B, o_lvt); t.h1_vt = at<uint16_t>(B, o_h1vt);
  t.lwall = at<uint32_t>(B, o_lw);
  h->bc_nodes = at<int32_t>(B, o_bcn);
  h->n_bc_nodes = h->L.bc_cells.empty() ? 0 : (int)P.bc_nodes.size();
  // the host copy of the plan is not needed after the upload
  P.halo = {}; P.h1_t3 = {}; P.h1_st = {}; P.lt3 = {}; P.lst = {}; P.lfe = {}; P.eloc = {}; P.be = {}; P.beloc = {};
  P.tnode = {}; P.tn_start = {}; P.tn_own = {}; P.tn_cells = {}; P.lvt = {}; P.h1_vt = {}; P.lwall = {};
  P.bc_nodes = {};
  h->tiles_ok = true;
  return configure_tiles(h);
}

int upload(StormFvtHandle* h) {
  HostLayout& L = h->L;
  const int T = L.T, N = L.N, K = h->opt.rkorder;
  const size_t T3 = 3 * (size_t)T, TK = (size_t)L.kst * T;
  const int nblk = (T + kRed - 1) / kRed;
  const size_t nbce = std::max(L.nbce, 1), nbdr = std::max(L.nbdr, 1), nwall = std::max(L.nwall, 1);
  const size_t nnz = std::max(L.n2t_nnz, 1), nts = std::max<size_t>(L.ts_t.size(), 1);
  Arena A;
  struct Up {
    size_t off;
    const void* src;
    size_t bytes;
  };
  std::vector<Up> ups;
  auto cpy = [&](const auto& vec, size_t n_alloc) {
    using V = typename std::decay<decltype(vec)>::type::value_type;
    size_t o = A.take(sizeof(V) * n_alloc);
    if (!vec.empty()) ups.push_back({o, vec.data(), sizeof(V) * vec.size()});
    return o;
  };
  // constant mesh data
  size_t o_area = cpy(L.area, T), o_perim = cpy(L.perim, T), o_xc = cpy(L.xc, T), o_yc = cpy(L.yc, T);
  size_t o_z = cpy(L.z, T), o_dzx = cpy(L.delz_x, T), o_dzy = cpy(L.delz_y, T), o_zmax = cpy(L.zmax, T);
  size_t o_cd = cpy(L.cd, T), o_la = cpy(L.lsq_a, T), o_lb = cpy(L.lsq_b, T), o_lc = cpy(L.lsq_c, T);
  size_t o_ld = cpy(L.lsq_det, T);
  const bool wind = !L.wcoef1.empty();
  size_t o_wc1 = wind ? cpy(L.wcoef1, T) : 0, o_wc2 = wind ? cpy(L.wcoef2, T) : 0;
  const size_t ncv = std::max(L.ncv, 1), ncvc = std::max<size_t>(L.cvc_cell.size(), 1);
  const size_t ncvt = std::max<size_t>(L.cv_head.size(), 1);
  size_t o_cvin = cpy(L.cv_in, ncv), o_cvn = cpy(L.cv_n, ncv), o_cvrx = cpy(L.cv_rx, ncv);
  size_t o_cvry = cpy(L.cv_ry, ncv), o_cvz = cpy(L.cv_zinv, ncv), o_cvh = cpy(L.cv_head, ncvt);
  size_t o_cvq = cpy(L.cv_q, ncvt), o_cvcc = cpy(L.cvc_cell, ncvc), o_cvco = cpy(L.cvc_code, ncvc);
  size_t o_cvsrc = A.take(sizeof(double) * ncv);
  size_t o_nst = cpy(L.nst, T), o_ford = cpy(L.forder, T), o_hvm = cpy(L.hvmask, T), o_fk = cpy(L.fkind, T3);
  // face kinds and references in summation order (static; see Dev::fko)
  std::vector<uint16_t> fko(T, 0);
  std::vector<int32_t> frefo(T3, 0);
  for (size_t c = 0; c < (size_t)T; c++)
    for (int t = 0; t < 3; t++) {
      const int j = (L.forder[c] >> (2 * t)) & 3;
      fko[c] |= (uint16_t)((L.fkind[(size_t)j * T + c] & 7) << (3 * t));
      frefo[(size_t)t * T + c] = L.fref[(size_t)j * T + c];
    }
  size_t o_fko = cpy(fko, T), o_frefo = cpy(frefo, T3);
  size_t o_vert = cpy(L.vert, T3), o_t3 = cpy(L.t2t3, T3), o_fref = cpy(L.fref, T3), o_sid = cpy(L.st_id, TK);
  size_t o_rcx = cpy(L.rc_x, T3), o_rcy = cpy(L.rc_y, T3), o_fnx = cpy(L.fnx, T3), o_fny = cpy(L.fny, T3);
  size_t o_flen = cpy(L.flen, T3), o_fz0 = cpy(L.fz0, T3);
  size_t o_sw = cpy(L.st_w, TK), o_sdx = cpy(L.st_dx, TK), o_sdy = cpy(L.st_dy, TK);
  size_t o_wp1 = cpy(L.wall_p1, nwall), o_wp2 = cpy(L.wall_p2, nwall);
  size_t o_zv = cpy(L.zvtx, N), o_nx = cpy(L.node_x, N), o_ny = cpy(L.node_y, N), o_n2w = cpy(L.n2t_w, nnz);
  size_t o_n2o = cpy(L.n2t_off, (size_t)N + 1), o_n2c = cpy(L.n2t_cell, nnz), o_nh = cpy(L.node_hbc, N);
  size_t o_bk = cpy(L.bdr_kind, nbdr), o_bs = cpy(L.bdr_slot, nbdr), o_bo = cpy(L.bdr_off, nbdr);
  size_t o_bcn = cpy(L.bdr_cnt, nbdr), o_bcc = cpy(L.bce_cell, nbce), o_bcs = cpy(L.bce_slot, nbce);
  size_t o_bnx = cpy(L.bce_nx, nbce), o_bny = cpy(L.bce_ny, nbce), o_btx = cpy(L.bce_tx, nbce);
  size_t o_bty = cpy(L.bce_ty, nbce), o_bl = cpy(L.bce_len, nbce), o_bz = cpy(L.bce_zmid, nbce);
  size_t o_tst = cpy(L.ts_t, nts), o_tsv = cpy(L.ts_v, nts);
  size_t o_csid = cpy(L.cell_sid, T), o_nsid = cpy(L.node_sid, N);
  size_t o_esid = cpy(L.edge_sid, std::max(L.ne, 1)), o_bsid = cpy(L.bdr_sid, nbdr);
  size_t o_bcl = cpy(L.bc_cells, std::max<size_t>(L.bc_cells.size(), 1));
  const bool rsavg = h->opt.rsavg_passes > 0;
  size_t o_rsc = cpy(L.rs_cells, std::max<size_t>(L.rs_cells.size(), 1));
  size_t o_phi = A.take(rsavg ? 8 * 3 * (size_t)T : 8), o_phi0 = A.take(rsavg ? 8 * 3 * (size_t)T : 8);
  const size_t ne1 = std::max(L.ne, 1);
  // edges with a cell that has an open-boundary face: the fused kernel hands their
  // fluxes to k_flux_bc through the edge-flux arrays
  std::vector<uint8_t> eslot = L.eslot;
  for (int32_t e = 0; e < L.ne; e++)
    if ((L.forder[L.eL[e]] & kOrderHasBc) || (L.forder[L.eR[e]] & kOrderHasBc)) eslot[e] |= kEdgeExport;
  // vertex minus centroid of each cell vertex (the differences bed_slope_STD forms)
  std::vector<double> vox(T3), voy(T3);
  for (size_t q = 0; q < T3; q++) {
    const int32_t c = (int32_t)(q % (size_t)T), v = L.vert[q];
    vox[q] = L.node_x[v] - L.xc[c];
    voy[q] = L.node_y[v] - L.yc[c];
  }
  size_t o_vox = cpy(vox, T3), o_voy = cpy(voy, T3);
  size_t o_eL = cpy(L.eL, ne1), o_eR = cpy(L.eR, ne1), o_es = cpy(eslot, ne1);
  size_t o_enx = cpy(L.enx, ne1), o_eny = cpy(L.eny, ne1), o_el = cpy(L.elen, ne1), o_ez0 = cpy(L.ez0, ne1);
  // state
  const size_t TL = (size_t)(K + 1) * T;
  size_t o_rkh = A.take(8 * TL), o_rku = A.take(8 * TL), o_rkv = A.take(8 * TL);
  size_t o_ua = A.take(8 * (size_t)T), o_va = A.take(8 * (size_t)T), o_vz = A.take((size_t)T);
  size_t o_ub = h->mixed ? A.take(8 * (size_t)T) : 0, o_vb = h->mixed ? A.take(8 * (size_t)T) : 0;
  size_t o_ua2 = A.take(8 * (size_t)T), o_va2 = A.take(8 * (size_t)T);
  size_t o_g[6];
  for (int i = 0; i < 6; i++) o_g[i] = A.take(8 * (size_t)T);
  size_t o_dra = A.take(T), o_drb = A.take(T), o_hv = A.take(8 * (size_t)N), o_vw = A.take(N);
  size_t o_dro = A.take(T);
  size_t o_pm = A.take(8 * (size_t)T), o_bcc3 = A.take(8 * 3 * nbce), o_rec = A.take(8 * 3 * nbce);
  size_t o_part = A.take(8 * 8 * (size_t)nblk), o_sc = A.take(sizeof(Scalars) * (size_t)h->nscen);
  size_t o_efx = A.take(8 * 3 * ne1), o_eok = A.take(ne1);
  cudaError_t e = cudaMalloc(&h->arena, A.off);
  if (e != cudaSuccess)
    return set_error(e == cudaErrorMemoryAllocation ? STORM_ERR_NOMEM : STORM_ERR_CUDA,
                     std::string("device allocation of ") + std::to_string(A.off) + " bytes: " + cudaGetErrorString(e));
  CK(cudaMemset(h->arena, 0, A.off));
  for (const Up& u : ups) CK(cudaMemcpy(static_cast<char*>(h->arena) + u.off, u.src, u.bytes, cudaMemcpyHostToDevice));
  void* B = h->arena;
  Dev& d = h->d;
  const StormFvtOptions& o = h->opt;
  d.T = T; d.N = N; d.K = K; d.kst = L.kst; d.nbdr = L.nbdr; d.nbce = L.nbce;
  d.steady = o.steady != 0; d.dt_op = o.dt_op; d.lim = o.opt_limiter; d.btype = o.btype;
  d.hvalve = o.hvalve != 0; d.vclip = o.vclip != 0; d.fric = o.opt_friction; d.stop_cr = o.stop_cr;
  d.flux = o.flux;
  d.h_dry = o.h_dry; d.h_wet = o.h_wet; d.cfl = o.cfl; d.vceiling = o.vceiling; d.visc = o.visc;
  d.rstop = o.rstop;
  // RK tables, dataprepFVT.f90:256-273
  std::memset(d.alpha, 0, sizeof d.alpha);
  std::memset(d.beta, 0, sizeof d.beta);
  if (K == 1) { d.alpha[1][0] = 1.0; d.beta[1] = 1.0; }
  if (K == 2) { d.alpha[1][0] = 1.0; d.beta[1] = 1.0; d.alpha[2][0] = 0.5; d.alpha[2][1] = 0.5; d.beta[2] = 0.5; }
  if (K == 3) {
    d.alpha[1][0] = 1.0;
    d.alpha[2][0] = 0.750; d.alpha[2][1] = 0.250;
    d.alpha[3][0] = 1.0 / 3.0; d.alpha[3][1] = 0.0; d.alpha[3][2] = 2.0 / 3.0;
    d.beta[1] = 1.0; d.beta[2] = 0.250; d.beta[3] = 2.0 / 3.0;
  }
  d.area = at<double>(B, o_area); d.perim = at<double>(B, o_perim); d.xc = at<double>(B, o_xc);
  d.yc = at<double>(B, o_yc); d.z = at<double>(B, o_z); d.delz_x = at<double>(B, o_dzx);
  d.delz_y = at<double>(B, o_dzy); d.zmax = at<double>(B, o_zmax); d.cd = at<double>(B, o_cd);
  d.lsq_a = at<double>(B, o_la); d.lsq_b = at<double>(B, o_lb); d.lsq_c = at<double>(B, o_lc);
  d.lsq_det = at<double>(B, o_ld);
  d.wcoef1 = wind ? at<double>(B, o_wc1) : nullptr;
  d.wcoef2 = wind ? at<double>(B, o_wc2) : nullptr;
  d.ncv = L.ncv; d.cv_ld = L.cv_ld; d.ncvc = (int32_t)L.cvc_cell.size();
  d.cv_in = at<int32_t>(B, o_cvin); d.cv_n = at<int32_t>(B, o_cvn); d.cv_rx = at<double>(B, o_cvrx);
  d.cv_ry = at<double>(B, o_cvry); d.cv_zinv = at<double>(B, o_cvz); d.cv_head = at<double>(B, o_cvh);
  d.cv_q = at<double>(B, o_cvq); d.cvc_cell = at<int32_t>(B, o_cvcc); d.cvc_code = at<int32_t>(B, o_cvco);
  d.cvsrc = at<double>(B, o_cvsrc);
  d.nst = at<uint8_t>(B, o_nst); d.forder = at<uint8_t>(B, o_ford); d.hvmask = at<uint8_t>(B, o_hvm);
  d.fkind = at<uint8_t>(B, o_fk);
  d.vert = at<int32_t>(B, o_vert); d.t2t3 = at<int32_t>(B, o_t3); d.fref = at<int32_t>(B, o_fref);
  d.fko = at<uint16_t>(B, o_fko); d.frefo = at<int32_t>(B, o_frefo);
  d.st_id = at<int32_t>(B, o_sid);
  d.rc_x = at<double>(B, o_rcx); d.rc_y = at<double>(B, o_rcy); d.fnx = at<double>(B, o_fnx);
  d.fny = at<double>(B, o_fny); d.flen = at<double>(B, o_flen); d.fz0 = at<double>(B, o_fz0);
  d.st_w = at<double>(B, o_sw); d.st_dx = at<double>(B, o_sdx); d.st_dy = at<double>(B, o_sdy);
  d.wall_p1 = at<int32_t>(B, o_wp1); d.wall_p2 = at<int32_t>(B, o_wp2);
  d.zvtx = at<double>(B, o_zv); d.node_x = at<double>(B, o_nx); d.node_y = at<double>(B, o_ny);
  d.n2t_w = at<double>(B, o_n2w); d.n2t_off = at<int32_t>(B, o_n2o); d.n2t_cell = at<int32_t>(B, o_n2c);
  d.node_hbc = at<int16_t>(B, o_nh);
  d.bdr_kind = at<int32_t>(B, o_bk); d.bdr_slot = at<int32_t>(B, o_bs); d.bdr_off = at<int32_t>(B, o_bo);
  d.bdr_cnt = at<int32_t>(B, o_bcn); d.bce_cell = at<int32_t>(B, o_bcc); d.bce_slot = at<int32_t>(B, o_bcs);
  d.bce_nx = at<double>(B, o_bnx); d.bce_ny = at<double>(B, o_bny); d.bce_tx = at<double>(B, o_btx);
  d.bce_ty = at<double>(B, o_bty); d.bce_len = at<double>(B, o_bl); d.bce_zmid = at<double>(B, o_bz);
  d.ts_t = at<double>(B, o_tst); d.ts_v = at<double>(B, o_tsv);
  d.cell_sid = at<int32_t>(B, o_csid); d.node_sid = at<int32_t>(B, o_nsid);
  d.edge_sid = at<int32_t>(B, o_esid); d.bdr_sid = at<int32_t>(B, o_bsid);
  d.nscen = h->nscen;
  d.t_real = h->nscen == 1 ? h->info[0].cell_cnt : T;
  d.lsq_derived = L.lsq_derived ? 1 : 0;
  d.rkh = at<double>(B, o_rkh); d.rku = at<double>(B, o_rku); d.rkv = at<double>(B, o_rkv);
  d.u_a = at<double>(B, o_ua); d.v_a = at<double>(B, o_va); d.vzero = at<uint8_t>(B, o_vz);
  d.u_b = h->mixed ? at<double>(B, o_ub) : nullptr;
  d.v_b = h->mixed ? at<double>(B, o_vb) : nullptr;
  h->u_a2 = at<double>(B, o_ua2); h->v_a2 = at<double>(B, o_va2);
  d.vox = at<double>(B, o_vox); d.voy = at<double>(B, o_voy);
  d.delh_x = at<double>(B, o_g[0]); d.delh_y = at<double>(B, o_g[1]); d.delu_x = at<double>(B, o_g[2]);
  d.delu_y = at<double>(B, o_g[3]); d.delv_x = at<double>(B, o_g[4]); d.delv_y = at<double>(B, o_g[5]);
  d.dry_a = at<uint8_t>(B, o_dra); d.dry_b = at<uint8_t>(B, o_drb); d.hvtx = at<double>(B, o_hv);
  d.dry_out = at<uint8_t>(B, o_dro);
  d.rs_cells = at<int32_t>(B, o_rsc); d.phi = at<double>(B, o_phi); d.phi0 = at<double>(B, o_phi0);
  d.rs_fac1 = 1.0 / (1.0 + o.rsavg_eps * 3.0);  // solverFVT.f90:59-60
  d.rs_fac2 = o.rsavg_eps / (1.0 + o.rsavg_eps * 3.0);
  d.vwet = at<uint8_t>(B, o_vw); d.phimax = at<double>(B, o_pm); d.bc_c = at<double>(B, o_bcc3);
  d.bc_rec = at<double>(B, o_rec); d.part = at<double>(B, o_part); d.nblk_red = nblk;
  d.sc = at<Scalars>(B, o_sc);
  d.nbc_cells = (int32_t)L.bc_cells.size();
  d.ne = L.ne;
  d.eL = at<int32_t>(B, o_eL); d.eR = at<int32_t>(B, o_eR); d.eslot = at<uint8_t>(B, o_es);
  d.enx = at<double>(B, o_enx); d.eny = at<double>(B, o_eny); d.elen = at<double>(B, o_el);
  d.ez0 = at<double>(B, o_ez0); d.efx = at<double>(B, o_efx); d.eok = at<uint8_t>(B, o_eok);
  // FP64 views of the arithmetic-type arrays
  Geo<double>& gd = h->gd;
  gd.rc_x = d.rc_x; gd.rc_y = d.rc_y; gd.st_w = d.st_w; gd.st_dx = d.st_dx; gd.st_dy = d.st_dy;
  gd.lsq_a = d.lsq_a; gd.lsq_b = d.lsq_b; gd.lsq_c = d.lsq_c; gd.lsq_det = d.lsq_det;
  gd.delz_x = d.delz_x; gd.delz_y = d.delz_y; gd.enx = d.enx; gd.eny = d.eny; gd.elen = d.elen;
  gd.vox = d.vox; gd.voy = d.voy;
  gd.delh_x = d.delh_x; gd.delh_y = d.delh_y; gd.delu_x = d.delu_x; gd.delu_y = d.delu_y;
  gd.delv_x = d.delv_x; gd.delv_y = d.delv_y; gd.efx = d.efx;
  // FP32 copies for the mixed-precision path: the gradients and edge fluxes reuse the
  // FP64 buffers (a float array fits in the same bytes)
  Geo<float>& gf = h->gf;
  gf.delh_x = reinterpret_cast<float*>(d.delh_x); gf.delh_y = reinterpret_cast<float*>(d.delh_y);
  gf.delu_x = reinterpret_cast<float*>(d.delu_x); gf.delu_y = reinterpret_cast<float*>(d.delu_y);
  gf.delv_x = reinterpret_cast<float*>(d.delv_x); gf.delv_y = reinterpret_cast<float*>(d.delv_y);
  gf.efx = reinterpret_cast<float*>(d.efx);
  if (h->mixed) {
    auto f32 = [&](const std::vector<double>& v) {
      std::vector<float> f(v.size());
      for (size_t i = 0; i < v.size(); i++) f[i] = (float)v[i];
      return f;
    };
    struct FCopy {
      const float** dst;
      std::vector<float> host;
    };
    std::vector<FCopy> fc;
    fc.push_back({&gf.rc_x, f32(L.rc_x)});
    fc.push_back({&gf.rc_y, f32(L.rc_y)});
    fc.push_back({&gf.st_w, f32(L.st_w)});
    fc.push_back({&gf.st_dx, f32(L.st_dx)});
    fc.push_back({&gf.st_dy, f32(L.st_dy)});
    fc.push_back({&gf.lsq_a, f32(L.lsq_a)});
    fc.push_back({&gf.lsq_b, f32(L.lsq_b)});
    fc.push_back({&gf.lsq_c, f32(L.lsq_c)});
    fc.push_back({&gf.lsq_det, f32(L.lsq_det)});
    fc.push_back({&gf.delz_x, f32(L.delz_x)});
    fc.push_back({&gf.delz_y, f32(L.delz_y)});
    fc.push_back({&gf.enx, f32(L.enx)});
    fc.push_back({&gf.eny, f32(L.eny)});
    fc.push_back({&gf.elen, f32(L.elen)});
    fc.push_back({&gf.vox, f32(vox)});
    fc.push_back({&gf.voy, f32(voy)});
    size_t total = 0;
    for (auto& c : fc) total += (c.host.size() * 4 + 255) & ~(size_t)255;
    cudaError_t ef = cudaMalloc(&h->arena32, std::max<size_t>(total, 256));
    if (ef != cudaSuccess) return set_error(STORM_ERR_NOMEM, std::string("device allocation (mixed): ") + cudaGetErrorString(ef));
    size_t off = 0;
    for (auto& c : fc) {
      float* p = reinterpret_cast<float*>(static_cast<char*>(h->arena32) + off);
      if (!c.host.empty()) CK(cudaMemcpy(p, c.host.data(), c.host.size() * 4, cudaMemcpyHostToDevice));
      *c.dst = p;
      off += (c.host.size() * 4 + 255) & ~(size_t)255;
    }
  }
  d.bc_cells = at<int32_t>(B, o_bcl);
  // per-scenario scalars: boundary values, series offsets, ranges
  std::vector<Scalars> s0(h->nscen);
  int32_t ts_base = 0;
  for (int sI = 0; sI < h->nscen; sI++) {
    const HostLayout& P = h->parts[sI];
    const ScenarioInfo& I = h->info[sI];
    Scalars& x = s0[sI];
    std::memset(&x, 0, sizeof x);
    x.n_in = P.n_in;
    x.n_out = P.n_out;
    for (int b = 0; b < P.n_in; b++) x.qin[b] = P.qin[b];
    for (int b = 0; b < P.n_out; b++) {
      x.hbc[b] = P.hbc[b];
      x.out_type[b] = P.out_type[b];
    }
    for (int b = 0; b < P.n_in; b++) {
      x.ts_off[b] = P.ts_off[b] + ts_base;
      x.ts_cnt[b] = P.ts_cnt[b];
    }
    for (int b = 0; b < P.n_out; b++) {
      x.ts_off[kMaxBdrDev + b] = P.ts_off[P.n_in + b] + ts_base;
      x.ts_cnt[kMaxBdrDev + b] = P.ts_cnt[P.n_in + b];
    }
    ts_base += (int32_t)P.ts_t.size();
    x.bch_max = P.bch_max;
    x.last_cell = I.last_cell;
    x.blk_off = I.blk_off;
    x.blk_cnt = I.blk_cnt;
  }
  CK(cudaMemcpy(d.sc, s0.data(), sizeof(Scalars) * s0.size(), cudaMemcpyHostToDevice));
  int rct = upload_tiles(h);
  if (rct) return rct;
  int maxcnt = 1;
  for (int b = 0; b < L.nbdr; b++) maxcnt = std::max(maxcnt, L.bdr_cnt[b]);
  // per edge: two sums' terms (16 B) and a flag; with the fixed point's invariants
  // cached, four more doubles and two flags (up to about 4,000 edges per boundary)
  const size_t plain = (size_t)maxcnt * 2 * sizeof(double) + (((size_t)maxcnt + 7) & ~(size_t)7);
  const size_t cached = (size_t)maxcnt * 6 * sizeof(double) + (((size_t)2 * maxcnt + 7) & ~(size_t)7);
  d.bc_cache = cached <= 200 * 1024;
  h->bc_smem = d.bc_cache ? cached : plain;
  if (h->bc_smem > 48 * 1024) set_bc_smem_limit((int)h->bc_smem);
  return 0;
}

// fn(i0, i1) over [0, n) in contiguous chunks on up to 8 host threads (one below
// 256k items): the state permutations of large meshes are memory-latency bound.
template <class F>
void par_chunks(size_t n, F fn) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = n < (size_t)1 << 18 ? 1 : std::min<size_t>(std::min(8u, hw), n >> 16);
  if (nt <= 1) {
    fn((size_t)0, n);
    return;
  }
  std::vector<std::thread> th;
  const size_t step = (n + nt - 1) / nt;
  size_t done = step;  // chunks [step, done) are covered by started threads
  try {
    for (size_t t = 1; t < nt; t++) {
      th.emplace_back(fn, std::min(n, t * step), std::min(n, (t + 1) * step));
      done = std::min(n, (t + 1) * step);
    }
  } catch (const std::system_error&) {  // no more threads: the caller's thread does the rest
  }
  fn((size_t)0, std::min(n, step));
  if (done < n) fn(done, n);
  for (auto& x : th) x.join();
}

// Pinned host staging of at least n doubles for the state transfers (page-locked
// memory copies at full PCIe/C2C speed and asynchronously); nullptr if it cannot be
// had, and the caller then stages in pageable memory.
double* io_buffer(StormFvtHandle* h, size_t n) {
  if (h->io_n >= n) return h->io_host;
  if (h->io_host) cudaFreeHost(h->io_host);
  h->io_host = nullptr;
  h->io_n = 0;
  void* p = nullptr;
  if (cudaMallocHost(&p, n * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  h->io_host = static_cast<double*>(p);
  h->io_n = n;
  return h->io_host;
}

}  // namespace

extern "C" {

const char* storm_fvt_last_error(void) { return g_err.c_str(); }

void storm_fvt_default_options(StormFvtOptions* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->h_dry = 0.001;
  o->h_wet = 0.001;
  o->cfl = 1.0;
  o->vceiling = 35.0;
  o->rstop = (double)1.0e-4f;
  const double t = 18.0;  // viscosity.f90 at temp = 18 C
  o->visc = (double)1.792e-6f / (1.0 + 0.0337 * t + 0.000221 * t * t);
  o->steady = 1;
  o->dt_op = 0;
  o->rkorder = 2;
  o->opt_limiter = 2;
  o->btype = 0;
  o->hvalve = 1;
  o->vclip = 0;
  o->opt_friction = 0;
  o->stop_cr = 0;
  o->flux = STORM_FLUX_ROE;
  o->precision = STORM_PREC_FP64;
  o->device = 0;
}

int storm_fvt_create_batch(const StormFvtMesh* const* meshes, int32_t n, const StormFvtOptions* opt,
                           StormFvtHandle** out) {
  clear_error();
  if (!meshes || !opt || !out || n < 1) return set_error(STORM_ERR_ARG, "storm_fvt_create: null argument or n < 1");
  *out = nullptr;
  for (int32_t i = 0; i < n; i++)
    if (!meshes[i]) return set_error(STORM_ERR_ARG, "storm_fvt_create: null mesh");
  int rc = check_options(*opt);
  if (rc) return rc;
  StormFvtHandle* h = new (std::nothrow) StormFvtHandle();
  if (!h) return set_error(STORM_ERR_NOMEM, "storm_fvt_create: out of memory");
  h->opt = *opt;
  h->device = opt->device;
  h->mixed = opt->precision == STORM_PREC_MIXED;
  if (h->mixed) h->bs_eflux = 128;
  h->nscen = n;
  try {
    h->parts.resize(n);
    for (int32_t i = 0; i < n && !rc; i++) rc = build_layout(*meshes[i], *opt, h->parts[i]);
    if (!rc) merge_layouts(h->parts, kRed, h->L, h->info);
  } catch (const std::bad_alloc&) {
    rc = set_error(STORM_ERR_NOMEM, "storm_fvt_create: host out of memory");
  }
  if (!rc) {
    // the kernels index the [rows][T] columns (stencil, faces, RK levels) in 32 bits
    const int64_t rows = std::max<int64_t>({(int64_t)h->L.kst, 3, (int64_t)opt->rkorder + 1});
    if (rows * (int64_t)h->L.T >= (int64_t)INT32_MAX)
      rc = set_error(STORM_ERR_UNSUPPORTED, "storm_fvt_create: " + std::to_string(h->L.T) +
                                                " cell slots exceed the 32-bit indexing of one handle (split the batch)");
  }
  if (rc) {
    delete h;
    return rc;
  }
  h->have_scen_state.assign(n, 0);
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    delete h;
    return set_error(STORM_ERR_CUDA, std::string("storm_fvt_create: no CUDA device: ") + cudaGetErrorString(e));
  }
  if (h->device < 0 || h->device >= ndev) {
    delete h;
    return set_error(STORM_ERR_ARG, "storm_fvt_create: device ordinal out of range");
  }
  e = cudaSetDevice(h->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
  for (int i = 0; i < 4 && e == cudaSuccess; i++) {
    e = cudaEventCreateWithFlags(&h->fork_ev[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->join_ev[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->eflux_ev[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
  if (e == cudaSuccess) e = cudaMallocHost(&h->sc_host, sizeof(Scalars) * (size_t)n);
  if (e != cudaSuccess) {
    release(h);
    return set_error(STORM_ERR_CUDA, std::string("storm_fvt_create: ") + cudaGetErrorString(e));
  }
  if ((rc = upload(h)) || (rc = capture_graph(h))) {
    std::string msg = g_err;
    release(h);
    return set_error(rc, msg);
  }
  *out = h;
  return STORM_OK;
}

int storm_fvt_create(const StormFvtMesh* mesh, const StormFvtOptions* opt, StormFvtHandle** out) {
  return storm_fvt_create_batch(&mesh, 1, opt, out);
}

int32_t storm_fvt_num_scenarios(const StormFvtHandle* h) { return h ? h->nscen : 0; }

int storm_fvt_set_scenario_state(StormFvtHandle* h, int32_t sid, const double* hh, const double* u, const double* v) {
  clear_error();
  if (!h || !hh || !u || !v) return set_error(STORM_ERR_ARG, "storm_fvt_set_state: null argument");
  if (sid < 0 || sid >= h->nscen) return set_error(STORM_ERR_ARG, "storm_fvt_set_state: scenario out of range");
  CK(cudaSetDevice(h->device));
  const HostLayout& P = h->parts[sid];
  const ScenarioInfo& I = h->info[sid];
  const int Ts = P.T;
  std::vector<double> pageable;
  double* buf = io_buffer(h, 3 * (size_t)Ts);
  if (!buf) {
    pageable.resize(3 * (size_t)Ts);
    buf = pageable.data();
  }
  par_chunks((size_t)Ts, [&](size_t c0, size_t c1) {
    for (size_t c = c0; c < c1; c++) {
      const int o = P.cell_old[c];
      buf[c] = hh[o];
      buf[Ts + c] = u[o];
      buf[2 * (size_t)Ts + c] = v[o];
    }
  });
  const Dev& d = h->d;
  CK(cudaMemcpyAsync(d.rkh + I.cell_off, buf, 8 * (size_t)Ts, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(d.u_a + I.cell_off, buf + Ts, 8 * (size_t)Ts, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(d.v_a + I.cell_off, buf + 2 * (size_t)Ts, 8 * (size_t)Ts, cudaMemcpyHostToDevice,
                     h->stream));
  k_init<<<I.blk_cnt, kRed, 0, h->stream>>>(d, I.cell_off);
  k_init_final<<<1, kRed, 0, h->stream>>>(d, sid);
  CK(cudaGetLastError());
  h->launches += 2;
  CK(cudaStreamSynchronize(h->stream));
  h->have_scen_state[sid] = 1;
  h->have_state = true;
  for (uint8_t f : h->have_scen_state) h->have_state = h->have_state && f;
  return STORM_OK;
}

int storm_fvt_set_state(StormFvtHandle* h, const double* hh, const double* u, const double* v) {
  if (h && h->nscen != 1)
    return set_error(STORM_ERR_ARG, "storm_fvt_set_state: batched handle, use storm_fvt_set_scenario_state");
  return storm_fvt_set_scenario_state(h, 0, hh, u, v);
}

static void fill_stats(const StormFvtHandle* h, const Scalars& s, StormFvtStepStats* stats) {
  std::memset(stats, 0, sizeof *stats);
  stats->iter = s.iter;
  stats->converged = s.converged;
  stats->ttime = s.ttime;
  stats->stime = s.stime;
  stats->delt = h->opt.steady ? s.delt_fric : s.delt;
  stats->rmax = s.rmax;
  stats->rms_dh = s.rms;
  stats->tmass = s.tmass;
  for (int b = 0; b < STORM_MAX_BDR; b++) {
    stats->cqin3[b] = s.cqin3[b];
    stats->cqout3[b] = s.cqout3[b];
  }
  stats->device_status = s.status;
}

int storm_fvt_step(StormFvtHandle* h, int32_t nsteps, StormFvtStepStats* stats) {
  clear_error();
  if (!h) return set_error(STORM_ERR_ARG, "storm_fvt_step: null handle");
  if (!h->have_state) return set_error(STORM_ERR_ARG, "storm_fvt_step: state not set");
  if (nsteps < 0) return set_error(STORM_ERR_ARG, "storm_fvt_step: negative step count");
  CK(cudaSetDevice(h->device));
  const int poll = h->opt.steady ? 16 : (1 << 30);
  const size_t scb = sizeof(Scalars) * (size_t)h->nscen;
  h->last_flux_ms = 0.0;
  h->last_flux_launches = 0;
  CK(cudaEventRecord(h->ev0, h->stream));
  if (h->timing) {
    const size_t need = 2 * (size_t)(h->kernels_per_step + 2) * nsteps;
    while (h->fev.size() < need) {
      cudaEvent_t ev;
      CK(cudaEventCreate(&ev));
      h->fev.push_back(ev);
    }
    h->fev_class.assign(need / 2, 0);
    size_t used = 0;
    for (int i = 0; i < nsteps; i++) {
      int rc = enqueue_step(h, true, &used);
      if (rc) return rc;
      h->launches += h->kernels_per_step;
    }
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < 8; c++) {
      h->kt_ms[c] = 0.0;
      h->kt_n[c] = 0;
    }
    for (size_t i = 0; i + 1 < used; i += 2) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, h->fev[i], h->fev[i + 1]));
      const int c = h->fev_class[i / 2];
      h->kt_ms[c] += ms;
      h->kt_n[c] += 1;
    }
    h->last_flux_ms = h->kt_ms[KT_FLUX];
    h->last_flux_launches = h->kt_n[KT_FLUX];
  } else {
    for (int i = 0; i < nsteps; i++) {
      CK(cudaGraphLaunch(h->exec, h->stream));
      h->launches += h->kernels_per_step;
      if ((i + 1) % poll == 0 && i + 1 < nsteps) {
        CK(cudaMemcpyAsync(h->sc_host, h->d.sc, scb, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        bool all = true;
        for (int sI = 0; sI < h->nscen; sI++) all = all && h->sc_host[sI].converged;
        if (all) break;
      }
    }
    CK(cudaEventRecord(h->ev1, h->stream));
  }
  CK(cudaMemcpyAsync(h->sc_host, h->d.sc, scb, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->last_step_ms = ms;
  if (stats) fill_stats(h, h->sc_host[0], stats);
  for (int sI = 0; sI < h->nscen; sI++)
    if (h->sc_host[sI].status & 1)
      return set_error(STORM_ERR_DEVICE, "storm_fvt_step: non-finite depth or velocity in scenario " +
                                             std::to_string(sI));
  return STORM_OK;
}

int storm_fvt_scenario_stats(const StormFvtHandle* h, int32_t sid, StormFvtStepStats* stats) {
  if (!h || !stats) return set_error(STORM_ERR_ARG, "storm_fvt_scenario_stats: null argument");
  if (sid < 0 || sid >= h->nscen) return set_error(STORM_ERR_ARG, "storm_fvt_scenario_stats: scenario out of range");
  fill_stats(h, h->sc_host[sid], stats);
  return STORM_OK;
}

int storm_fvt_get_scenario_state(StormFvtHandle* h, int32_t sid, double* hh, double* u, double* v, double* rkh,
                                 double* rku, double* rkv, double* hvtx) {
  clear_error();
  if (!h) return set_error(STORM_ERR_ARG, "storm_fvt_get_state: null handle");
  if (sid < 0 || sid >= h->nscen) return set_error(STORM_ERR_ARG, "storm_fvt_get_state: scenario out of range");
  CK(cudaSetDevice(h->device));
  const HostLayout& P = h->parts[sid];
  const ScenarioInfo& I = h->info[sid];
  const int Ts = P.T, Ns = P.N;
  const size_t m = (size_t)std::max(Ts, Ns);
  // up to three arrays per round trip: their copies are issued together into the
  // staging buffer, then each is permuted back to the caller's element order
  std::vector<double> pageable;
  double* buf = io_buffer(h, 3 * m);
  if (!buf) {
    pageable.resize(3 * m);
    buf = pageable.data();
  }
  struct Pull {
    const double* dev;
    double* dst;
    int n;
    const std::vector<int32_t>* perm;
  };
  auto round = [&](std::initializer_list<Pull> items) -> int {
    size_t k = 0;
    for (const Pull& it : items)
      if (it.dst) CK(cudaMemcpyAsync(buf + (k++) * m, it.dev, 8 * (size_t)it.n, cudaMemcpyDeviceToHost, h->stream));
    if (k == 0) return 0;
    CK(cudaStreamSynchronize(h->stream));
    k = 0;
    for (const Pull& it : items) {
      if (!it.dst) continue;
      const double* src = buf + (k++) * m;
      par_chunks((size_t)it.n, [&](size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; i++) it.dst[(*it.perm)[i]] = src[i];
      });
    }
    return 0;
  };
  const Dev& d = h->d;
  const int co = I.cell_off, no = I.node_off;
  int rc;
  if ((rc = round({{d.rkh + co, hh, Ts, &P.cell_old}, {d.u_a + co, u, Ts, &P.cell_old},
                   {d.v_a + co, v, Ts, &P.cell_old}})))
    return rc;
  if ((rc = round({{d.rkh + co, rkh, Ts, &P.cell_old}, {d.rku + co, rku, Ts, &P.cell_old},
                   {d.rkv + co, rkv, Ts, &P.cell_old}})))
    return rc;
  if ((rc = round({{d.hvtx + no, hvtx, Ns, &P.node_old}}))) return rc;
  return STORM_OK;
}

int storm_fvt_get_state(StormFvtHandle* h, double* hh, double* u, double* v, double* rkh, double* rku, double* rkv,
                        double* hvtx) {
  if (h && h->nscen != 1)
    return set_error(STORM_ERR_ARG, "storm_fvt_get_state: batched handle, use storm_fvt_get_scenario_state");
  return storm_fvt_get_scenario_state(h, 0, hh, u, v, rkh, rku, rkv, hvtx);
}

int storm_fvt_output_vertices(StormFvtHandle* h, const StormFvtOutputBoundary* ob, int32_t in_loop, double* hvtx,
                              double* uvtx, double* vvtx, double* cdvtx, double* e_est) {
  clear_error();
  if (!h || !ob) return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: null argument");
  if (h->nscen != 1) return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: batched handle");
  if (!h->have_state) return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: state not set");
  if (h->d.K < 2)
    return set_error(STORM_ERR_UNSUPPORTED, "storm_fvt_output_vertices: needs rkorder >= 2 (the last stage's input)");
  CK(cudaSetDevice(h->device));
  const HostLayout& P = h->parts[0];
  const int N = P.N, T = P.T;
  const Scalars& sc = h->sc_host[0];  // boundary values of the last completed iteration
  // boundary lists in the device numbering
  std::vector<int32_t> iv;   // wall nodes | outflow nodes | out_off | out_type | inflow nodes | in_off | in_type
  std::vector<double> dv;    // wtang | hn | hbc | pn | lin | qin | qin2
  if (ob->n_wall < 0 || (ob->n_wall > 0 && (!ob->wall_pts || !ob->wtangs)))
    return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: wall arrays missing");
  auto node_of = [&](int32_t p, int32_t* out) -> bool {
    if (p < 1 || p > N) return false;
    *out = P.node_new[p - 1];
    return true;
  };
  const size_t i_wall = iv.size();
  for (int32_t i = 0; i < ob->n_wall; i++) {
    int32_t q;
    if (!node_of(ob->wall_pts[i], &q)) return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: wall node out of range");
    iv.push_back(q);
  }
  const size_t d_wt = dv.size();
  for (int32_t i = 0; i < 2 * ob->n_wall; i++) dv.push_back(ob->wtangs[i]);
  const int n_out = P.n_out;
  const size_t i_onode = iv.size();
  iv.insert(iv.end(), P.out_node.begin(), P.out_node.end());
  const size_t i_ooff = iv.size();
  iv.insert(iv.end(), P.out_off.begin(), P.out_off.end());
  const size_t i_otype = iv.size();
  for (int b = 0; b < n_out; b++) iv.push_back(P.out_type[b]);
  const size_t d_hn = dv.size();
  if (n_out > 0 && (!ob->hnormals || ob->hbc_ld < 1))
    return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: hnormals missing");
  for (int b = 0; b < n_out; b++)
    for (int i = 0; i < P.out_off[b + 1] - P.out_off[b]; i++) {
      if (i >= ob->hbc_ld) return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: hbc_ld too small");
      dv.push_back(ob->hnormals[2 * ((size_t)b * ob->hbc_ld + i)]);
      dv.push_back(ob->hnormals[2 * ((size_t)b * ob->hbc_ld + i) + 1]);
    }
  const size_t d_hbc = dv.size();
  for (int b = 0; b < n_out; b++) dv.push_back(in_loop ? sc.hbc_it[b] : sc.hbc[b]);
  const int n_in = P.n_in;
  if (n_in > 0 && (!ob->n_qin || !ob->qin_nodes || !ob->pnormals || !ob->l_inflow || ob->qin_ld < 1))
    return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: inflow arrays missing");
  const size_t i_inode = iv.size();
  std::vector<int32_t> in_off(1, 0);
  const size_t d_pn0 = dv.size();
  std::vector<double> pn, lin;
  for (int b = 0; b < n_in; b++) {
    const int32_t n = ob->n_qin[b];
    if (n < 0 || n > ob->qin_ld) return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: n_qin out of range");
    for (int32_t i = 0; i < n; i++) {
      int32_t q;
      if (!node_of(ob->qin_nodes[(size_t)b * ob->qin_ld + i], &q))
        return set_error(STORM_ERR_ARG, "storm_fvt_output_vertices: inflow node out of range");
      iv.push_back(q);
      pn.push_back(ob->pnormals[2 * ((size_t)b * ob->qin_ld + i)]);
      pn.push_back(ob->pnormals[2 * ((size_t)b * ob->qin_ld + i) + 1]);
      lin.push_back(ob->l_inflow[(size_t)b * ob->qin_ld + i]);
    }
    in_off.push_back(in_off.back() + n);
  }
  (void)d_pn0;
  const size_t i_ioff = iv.size();
  iv.insert(iv.end(), in_off.begin(), in_off.end());
  const size_t i_itype = iv.size();
  for (int b = 0; b < n_in; b++) iv.push_back(P.in_type[b]);
  const size_t d_pn = dv.size();
  dv.insert(dv.end(), pn.begin(), pn.end());
  const size_t d_lin = dv.size();
  dv.insert(dv.end(), lin.begin(), lin.end());
  const size_t d_qin = dv.size();
  for (int b = 0; b < n_in; b++) dv.push_back(in_loop ? sc.qin_it[b] : sc.qin[b]);
  const size_t d_qin2 = dv.size();
  for (int b = 0; b < n_in; b++) dv.push_back(ob->qin2 ? ob->qin2[b] : 0.0);
  iv.push_back(0);
  dv.push_back(0.0);
  // device buffer: outputs (hv, uv, vv, cdv [N], e_est [T]) then the lists
  const size_t out_d = 8 * (4 * (size_t)h->d.N + (size_t)h->d.T);
  const size_t need = out_d + 8 * dv.size() + 4 * iv.size() + 256;
  if (need > h->out_bytes) {
    if (h->out_buf) cudaFree(h->out_buf);
    h->out_buf = nullptr;
    h->out_bytes = 0;
    cudaError_t e = cudaMalloc(&h->out_buf, need);
    if (e != cudaSuccess) return set_error(STORM_ERR_NOMEM, "storm_fvt_output_vertices: device allocation failed");
    h->out_bytes = need;
  }
  char* base = static_cast<char*>(h->out_buf);
  double* dd = reinterpret_cast<double*>(base + out_d);
  int32_t* di = reinterpret_cast<int32_t*>(base + out_d + 8 * dv.size());
  CK(cudaMemcpyAsync(dd, dv.data(), 8 * dv.size(), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(di, iv.data(), 4 * iv.size(), cudaMemcpyHostToDevice, h->stream));
  OutputArgs a{};
  a.hv = reinterpret_cast<double*>(base);
  a.uv = a.hv + h->d.N;
  a.vv = a.uv + h->d.N;
  a.cdv = a.vv + h->d.N;
  a.e_est = a.cdv + h->d.N;
  a.n_out = n_out;
  a.out_node = di + i_onode; a.out_off = di + i_ooff; a.out_type = di + i_otype;
  a.hn = dd + d_hn; a.hbc = dd + d_hbc;
  a.n_wall = ob->n_wall; a.wall_node = di + i_wall; a.wtang = dd + d_wt;
  a.n_in = n_in;
  a.in_node = di + i_inode; a.in_off = di + i_ioff; a.in_type = di + i_itype;
  a.pn = dd + d_pn; a.lin = dd + d_lin; a.qin = dd + d_qin; a.qin2 = dd + d_qin2;
  launch_output(h->d, h->gd, h->gf, h->mixed, a, h->stream);
  h->launches += 4 + (n_out > 0) + (ob->n_wall > 0) + (n_in > 0) + ((!h->opt.steady && h->opt.dt_op == 1) ? 2 : 0);
  CK(cudaGetLastError());
  // results in element / node order
  std::vector<double> buf(std::max(N, T));
  auto pull = [&](const double* dev, double* dst, int n, const std::vector<int32_t>& perm) -> int {
    if (!dst) return 0;
    CK(cudaMemcpyAsync(buf.data(), dev, 8 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < n; k++) dst[perm[k]] = buf[k];
    return 0;
  };
  int rc;
  if ((rc = pull(a.hv, hvtx, N, P.node_old)) || (rc = pull(a.uv, uvtx, N, P.node_old)) ||
      (rc = pull(a.vv, vvtx, N, P.node_old)) || (rc = pull(a.cdv, cdvtx, N, P.node_old)) ||
      (rc = pull(a.e_est, e_est, T, P.cell_old)))
    return rc;
  CK(cudaStreamSynchronize(h->stream));
  return STORM_OK;
}

int storm_fvt_get_drycell(StormFvtHandle* h, int32_t* dry) {
  clear_error();
  if (!h || !dry) return set_error(STORM_ERR_ARG, "storm_fvt_get_drycell: null argument");
  if (h->nscen != 1) return set_error(STORM_ERR_ARG, "storm_fvt_get_drycell: batched handle");
  CK(cudaSetDevice(h->device));
  const HostLayout& P = h->parts[0];
  const int Ts = P.T;
  std::vector<uint8_t> b(Ts);
  CK(cudaMemcpyAsync(b.data(), h->d.dry_a, Ts, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int c = 0; c < Ts; c++) dry[P.cell_old[c]] = b[c] ? 1 : 0;
  return STORM_OK;
}

int64_t storm_fvt_kernel_launches(const StormFvtHandle* h) { return h ? h->launches : 0; }

int storm_fvt_set_kernel_timing(StormFvtHandle* h, int32_t on) {
  if (!h) return set_error(STORM_ERR_ARG, "storm_fvt_set_kernel_timing: null handle");
  h->timing = on != 0;
  return STORM_OK;
}

int storm_fvt_last_timing(const StormFvtHandle* h, double* step_ms, double* flux_ms, int64_t* flux_launches) {
  if (!h) return set_error(STORM_ERR_ARG, "storm_fvt_last_timing: null handle");
  if (step_ms) *step_ms = h->last_step_ms;
  if (flux_ms) *flux_ms = h->last_flux_ms;
  if (flux_launches) *flux_launches = h->last_flux_launches;
  return STORM_OK;
}

int storm_fvt_kernel_times(const StormFvtHandle* h, double* ms, int64_t* launches) {
  if (!h || !ms || !launches) return set_error(STORM_ERR_ARG, "storm_fvt_kernel_times: null argument");
  for (int c = 0; c < 8; c++) {
    ms[c] = h->kt_ms[c];
    launches[c] = h->kt_n[c];
  }
  return STORM_OK;
}

int storm_fvt_autotune(StormFvtHandle* h, int32_t iters, int32_t* chosen) {
  clear_error();
  if (!h) return set_error(STORM_ERR_ARG, "storm_fvt_autotune: null handle");
  if (!h->have_state) return set_error(STORM_ERR_ARG, "storm_fvt_autotune: state not set");
  if (iters < 1) iters = 1;
  CK(cudaSetDevice(h->device));
  // snapshot of the mutable state (restored afterwards: tuning does not advance the run)
  const Dev& d = h->d;
  const size_t T = (size_t)d.T, L = (size_t)(d.K + 1) * T;
  const size_t bytes = 8 * (3 * L + 2 * T) + 2 * T + sizeof(Scalars) * (size_t)h->nscen;
  char* snap = nullptr;
  CK(cudaMalloc(&snap, bytes));
  struct Piece {
    void* p;
    size_t n;
  } pieces[] = {{d.rkh, 8 * L}, {d.rku, 8 * L}, {d.rkv, 8 * L}, {d.u_a, 8 * T}, {d.v_a, 8 * T},
                {d.dry_a, T}, {d.dry_b, T}, {d.sc, sizeof(Scalars) * (size_t)h->nscen}};
  size_t off = 0;
  for (auto& pc : pieces) {
    CK(cudaMemcpyAsync(snap + off, pc.p, pc.n, cudaMemcpyDeviceToDevice, h->stream));
    off += pc.n;
  }
  // the stage path first: whole iterations (graph replays) of each path, from the same
  // state, the fastest kept
  auto restore = [&]() -> int {
    size_t o2 = 0;
    for (auto& pc : pieces) {
      CK(cudaMemcpyAsync(pc.p, snap + o2, pc.n, cudaMemcpyDeviceToDevice, h->stream));
      o2 += pc.n;
    }
    CK(cudaStreamSynchronize(h->stream));
    return 0;
  };
  int rc = 0;
  {
    const bool want0 = h->want_tiles, nodes0 = h->fuse_nodes;
    int best_path = -1;
    double best_ms = 1e300;
    const int paths[3] = {STORM_STAGE_PHASES, STORM_STAGE_FUSED, STORM_STAGE_FUSED_NODE_KERNEL};
    for (int p : paths) {
      if (p != STORM_STAGE_PHASES && !h->tiles_ok) continue;
      if ((rc = storm_fvt_set_stage_path(h, p))) break;
      if (p != STORM_STAGE_PHASES && storm_fvt_stage_path(h) != p) continue;  // not applicable here
      if ((rc = restore()) || (rc = storm_fvt_step(h, iters, nullptr))) break;
      if (h->last_step_ms < best_ms) {
        best_ms = h->last_step_ms;
        best_path = p;
      }
    }
    if (!rc && (rc = restore())) {}
    if (!rc) rc = storm_fvt_set_stage_path(h, best_path >= 0 ? best_path : (want0 ? (nodes0 ? 1 : 2) : 0));
    if (rc) {
      cudaFree(snap);
      return rc;
    }
  }
  struct Knob {
    int* bs;
    int cls;
    int cand[3];
  } knobs[] = {{&h->bs_node, KT_NODE, {64, 128, 256}},
               {&h->bs_grad, KT_GRAD, {64, 128, 256}},
               {&h->bs_eflux, KT_EFLUX, {32, 64, 128}},
               {&h->bs_flux, KT_FLUX, {32, 64, 128}}};
  const bool was_timing = h->timing;
  h->timing = true;
  for (auto& kb : knobs) {
    double best = 1e300;
    int best_bs = *kb.bs;
    for (int cand : kb.cand) {
      *kb.bs = cand;
      if ((rc = storm_fvt_step(h, iters, nullptr))) break;
      const double t = h->kt_ms[kb.cls];
      if (t < best) {
        best = t;
        best_bs = cand;
      }
    }
    *kb.bs = best_bs;
    if (rc) break;
  }
  h->timing = was_timing;
  off = 0;
  for (auto& pc : pieces) {
    cudaMemcpyAsync(pc.p, snap + off, pc.n, cudaMemcpyDeviceToDevice, h->stream);
    off += pc.n;
  }
  cudaStreamSynchronize(h->stream);
  cudaFree(snap);
  if (rc) return rc;
  if (chosen) {
    chosen[0] = h->bs_node;
    chosen[1] = h->bs_grad;
    chosen[2] = h->bs_eflux;
    chosen[3] = h->bs_flux;
  }
  // re-capture the iteration graph with the chosen shapes
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->exec = nullptr;
  h->graph = nullptr;
  return capture_graph(h);
}

int storm_fvt_set_stage_path(StormFvtHandle* h, int32_t path) {
  clear_error();
  if (!h) return set_error(STORM_ERR_ARG, "storm_fvt_set_stage_path: null handle");
  if (path != STORM_STAGE_PHASES && path != STORM_STAGE_FUSED && path != STORM_STAGE_FUSED_NODE_KERNEL)
    return set_error(STORM_ERR_ARG, "storm_fvt_set_stage_path: unknown path");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  h->want_tiles = path != STORM_STAGE_PHASES;
  h->fuse_nodes = path == STORM_STAGE_FUSED;
  if (h->tiles_ok) {
    int rc = configure_tiles(h);
    if (rc) return rc;
  }
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->exec = nullptr;
  h->graph = nullptr;
  return capture_graph(h);
}

int32_t storm_fvt_stage_path(const StormFvtHandle* h) {
  if (!h || !h->use_tiles) return STORM_STAGE_PHASES;
  return h->td.nodes ? STORM_STAGE_FUSED : STORM_STAGE_FUSED_NODE_KERNEL;
}

// ---- one part of a mesh per process ------------------------------------------------

static int part_handle(StormFvtHandle* h, const char* who) {
  if (!h) return set_error(STORM_ERR_ARG, std::string(who) + ": null handle");
  if (h->nscen != 1 || h->d.linked) return set_error(STORM_ERR_ARG, std::string(who) + ": needs a single-mesh handle");
  if (!h->have_state) return set_error(STORM_ERR_ARG, std::string(who) + ": state not set");
  CK(cudaSetDevice(h->device));
  return 0;
}

static int read_scalars(StormFvtHandle* h) {
  CK(cudaMemcpyAsync(h->sc_host, h->d.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int storm_fvt_set_exchange(StormFvtHandle* h, int32_t n_send, const int32_t* send_elems, int32_t n_recv,
                           const int32_t* recv_elems) {
  clear_error();
  if (!h) return set_error(STORM_ERR_ARG, "storm_fvt_set_exchange: null handle");
  if (h->nscen != 1 || h->d.linked) return set_error(STORM_ERR_ARG, "storm_fvt_set_exchange: needs a single-mesh handle");
  if (n_send < 0 || n_recv < 0 || (n_send && !send_elems) || (n_recv && !recv_elems))
    return set_error(STORM_ERR_ARG, "storm_fvt_set_exchange: bad element lists");
  const HostLayout& P = h->parts[0];
  const int32_t T = h->d.T;
  std::vector<int32_t> ss(std::max(n_send, 1)), rs(std::max(n_recv, 1));
  std::vector<uint8_t> mask(T, 0);
  for (int32_t i = 0; i < n_send; i++) {
    if (send_elems[i] < 1 || send_elems[i] > P.T) return set_error(STORM_ERR_ARG, "storm_fvt_set_exchange: element out of range");
    ss[i] = P.cell_new[send_elems[i] - 1];
  }
  for (int32_t i = 0; i < n_recv; i++) {
    if (recv_elems[i] < 1 || recv_elems[i] > P.T) return set_error(STORM_ERR_ARG, "storm_fvt_set_exchange: element out of range");
    rs[i] = P.cell_new[recv_elems[i] - 1];
    if (mask[rs[i]]) return set_error(STORM_ERR_ARG, "storm_fvt_set_exchange: a received element is listed twice");
    mask[rs[i]] = 1;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  if (h->xchg_buf) cudaFree(h->xchg_buf);
  h->xchg_buf = nullptr;
  const size_t a = (4 * ss.size() + 255) & ~(size_t)255, b = (4 * rs.size() + 255) & ~(size_t)255;
  cudaError_t e = cudaMalloc(&h->xchg_buf, a + b + T);
  if (e != cudaSuccess) return set_error(STORM_ERR_NOMEM, std::string("storm_fvt_set_exchange: ") + cudaGetErrorString(e));
  char* B = static_cast<char*>(h->xchg_buf);
  CK(cudaMemcpy(B, ss.data(), 4 * ss.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B + a, rs.data(), 4 * rs.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B + a + b, mask.data(), T, cudaMemcpyHostToDevice));
  h->send_slots = reinterpret_cast<int32_t*>(B);
  h->recv_slots = reinterpret_cast<int32_t*>(B + a);
  h->n_send = n_send;
  h->n_recv = n_recv;
  // the received (halo) cells stay out of this part's reductions
  h->d.halo_mask = reinterpret_cast<uint8_t*>(B + a + b);
  h->d.nhalo = n_recv;
  return 0;
}

int storm_fvt_iter_begin(StormFvtHandle* h, double* dt_local) {
  clear_error();
  int rc = part_handle(h, "storm_fvt_iter_begin");
  if (rc) return rc;
  if (!dt_local) return set_error(STORM_ERR_ARG, "storm_fvt_iter_begin: null argument");
  if ((rc = read_scalars(h))) return rc;
  *dt_local = h->sc_host[0].delt;
  return 0;
}

int storm_fvt_iter_set_dt(StormFvtHandle* h, double dt) {
  clear_error();
  int rc = part_handle(h, "storm_fvt_iter_set_dt");
  if (rc) return rc;
  if (!h->opt.steady) launch_part_scalar(h->d, 0, dt, h->stream);
  CK(cudaGetLastError());
  return 0;
}

int storm_fvt_iter_stage(StormFvtHandle* h, int32_t s, double* delt_last) {
  clear_error();
  int rc = part_handle(h, "storm_fvt_iter_stage");
  if (rc) return rc;
  if (s < 1 || s > h->d.K) return set_error(STORM_ERR_ARG, "storm_fvt_iter_stage: stage out of range");
  size_t dummy = 0;
  if ((rc = enqueue_step(h, false, &dummy, s))) return rc;
  h->launches += h->kernels_per_step / std::max(1, h->d.K);
  if ((rc = read_scalars(h))) return rc;
  if (delt_last) *delt_last = h->opt.steady ? h->sc_host[0].delt_fric : h->sc_host[0].delt;
  return 0;
}

int storm_fvt_iter_fric(StormFvtHandle* h, double delt, double* sums) {
  clear_error();
  int rc = part_handle(h, "storm_fvt_iter_fric");
  if (rc) return rc;
  if (!sums) return set_error(STORM_ERR_ARG, "storm_fvt_iter_fric: null argument");
  if (h->opt.steady) launch_part_scalar(h->d, 1, delt, h->stream);
  size_t dummy = 0;
  if ((rc = enqueue_step(h, false, &dummy, 0))) return rc;
  h->launches += 2;
  if ((rc = read_scalars(h))) return rc;
  const Scalars& sc = h->sc_host[0];
  sums[0] = sc.sumtop;
  sums[1] = sc.sumbot;
  sums[2] = sc.tmass;
  sums[3] = sc.rmax_phi;
  return 0;
}

int storm_fvt_iter_finish(StormFvtHandle* h, const double* sums, StormFvtStepStats* stats) {
  clear_error();
  int rc = part_handle(h, "storm_fvt_iter_finish");
  if (rc) return rc;
  if (!sums) return set_error(STORM_ERR_ARG, "storm_fvt_iter_finish: null argument");
  launch_part_finish(h->d, sums, h->stream);
  h->launches += 1;
  CK(cudaGetLastError());
  if ((rc = read_scalars(h))) return rc;
  if (stats) fill_stats(h, h->sc_host[0], stats);
  return 0;
}

// velocity buffers and dry flags of the state after stage `level` (after_fric = 0) or
// after the friction step (level 0)
static void part_buffers(StormFvtHandle* h, int level, int after_fric, double** u, double** v, uint8_t** dry) {
  const Dev& d = h->d;
  if (after_fric || !h->use_tiles) {
    *u = d.u_a;
    *v = d.v_a;
  } else {
    *u = (level & 1) ? h->u_a2 : d.u_a;
    *v = (level & 1) ? h->v_a2 : d.v_a;
  }
  *dry = after_fric ? d.dry_a : ((level & 1) ? d.dry_b : d.dry_a);
}

int storm_fvt_pack_halo(StormFvtHandle* h, int32_t level, int32_t after_fric, double* dev_out) {
  clear_error();
  int rc = part_handle(h, "storm_fvt_pack_halo");
  if (rc) return rc;
  if (level < 0 || level > h->d.K || (after_fric && level != 0))
    return set_error(STORM_ERR_ARG, "storm_fvt_pack_halo: level out of range (0 after the friction step)");
  if (h->n_send > 0 && !dev_out) return set_error(STORM_ERR_ARG, "storm_fvt_pack_halo: null buffer");
  double *u, *v;
  uint8_t* dry;
  part_buffers(h, level, after_fric, &u, &v, &dry);
  launch_pack(h->d, level, h->n_send, h->send_slots, u, v, dev_out, h->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int storm_fvt_unpack_halo(StormFvtHandle* h, int32_t level, int32_t after_fric, const double* dev_in) {
  clear_error();
  int rc = part_handle(h, "storm_fvt_unpack_halo");
  if (rc) return rc;
  if (level < 0 || level > h->d.K || (after_fric && level != 0))
    return set_error(STORM_ERR_ARG, "storm_fvt_unpack_halo: level out of range (0 after the friction step)");
  if (h->n_recv > 0 && !dev_in) return set_error(STORM_ERR_ARG, "storm_fvt_unpack_halo: null buffer");
  double *u, *v;
  uint8_t* dry;
  part_buffers(h, level, after_fric, &u, &v, &dry);
  launch_unpack(h->d, level, h->n_recv, h->recv_slots, dev_in, u, v, dry, h->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int storm_fvt_tile_check(const StormFvtMesh* const* meshes, int32_t n, int32_t tile_cells, int64_t* stats) {
  clear_error();
  if (!meshes || n < 1 || !stats || tile_cells < 32 || tile_cells > 4096)
    return set_error(STORM_ERR_ARG, "storm_fvt_tile_check: bad argument");
  StormFvtOptions o;
  storm_fvt_default_options(&o);
  std::vector<HostLayout> parts(n);
  std::vector<ScenarioInfo> info;
  HostLayout L;
  TilePlan P;
  try {
    for (int32_t i = 0; i < n; i++) {
      if (!meshes[i]) return set_error(STORM_ERR_ARG, "storm_fvt_tile_check: null mesh");
      int rc = build_layout(*meshes[i], o, parts[i]);
      if (rc) return rc;
    }
    merge_layouts(parts, kRed, L, info);
    if (build_tiles(L, tile_cells, P) != 0) return set_error(STORM_ERR_UNSUPPORTED, "storm_fvt_tile_check: tile too large");
  } catch (const std::bad_alloc&) {
    return set_error(STORM_ERR_NOMEM, "storm_fvt_tile_check: host out of memory");
  }
  int64_t s1 = 0, s2 = 0;
  for (int32_t t = 0; t < P.ntiles; t++) {
    s1 += P.info[(size_t)t * TI_N + TI_N1];
    s2 += P.info[(size_t)t * TI_N + TI_N2];
  }
  stats[0] = P.ntiles;
  stats[1] = P.ns_max;
  stats[2] = P.ng_max;
  stats[3] = P.ne_max;
  stats[4] = s1;
  stats[5] = s2;
  stats[6] = (int64_t)P.be.size();
  stats[7] = check_tiles(L, P);
  return 0;
}

int storm_fvt_link_partitions(StormFvtHandle* h, int32_t n_halo, const int32_t* dst_scen, const int32_t* dst_elem,
                              const int32_t* src_scen, const int32_t* src_elem, int32_t fric_scen) {
  clear_error();
  if (!h) return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: null handle");
  if (h->nscen < 2) return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: needs a batch of at least 2 parts");
  if (h->d.linked) return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: already linked");
  if (h->opt.rsavg_passes > 0)
    return set_error(STORM_ERR_UNSUPPORTED, "storm_fvt_link_partitions: residual smoothing is not supported");
  if (h->L.ncv > 0) return set_error(STORM_ERR_UNSUPPORTED, "storm_fvt_link_partitions: culverts are not supported");
  if (n_halo < 0 || (n_halo > 0 && (!dst_scen || !dst_elem || !src_scen || !src_elem)))
    return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: bad halo arrays");
  if (fric_scen < 0 || fric_scen >= h->nscen) return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: fric_scen out of range");
  const int T = h->L.T;
  auto slot = [&](int32_t s, int32_t e, int32_t* out) -> bool {
    if (s < 0 || s >= h->nscen) return false;
    const HostLayout& P = h->parts[s];
    if (e < 1 || e > P.T) return false;
    *out = h->info[s].cell_off + P.cell_new[e - 1];
    return true;
  };
  std::vector<int32_t> dst(n_halo), src(n_halo);
  std::vector<uint8_t> mask(T, 0);
  for (int32_t i = 0; i < n_halo; i++) {
    if (!slot(dst_scen[i], dst_elem[i], &dst[i]) || !slot(src_scen[i], src_elem[i], &src[i]))
      return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: halo entry " + std::to_string(i) + " out of range");
    if (dst_scen[i] == src_scen[i]) return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: a halo cell's owner is in its own part");
    if (mask[dst[i]]) return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: halo cell listed twice");
    mask[dst[i]] = 1;
  }
  for (int32_t i = 0; i < n_halo; i++)
    if (mask[src[i]]) return set_error(STORM_ERR_ARG, "storm_fvt_link_partitions: an owner is itself a halo cell");
  CK(cudaSetDevice(h->device));
  const size_t nh = std::max<int32_t>(n_halo, 1);
  const size_t o_dst = 0, o_src = (nh * 4 + 255) & ~(size_t)255, o_mask = o_src + ((nh * 4 + 255) & ~(size_t)255);
  const size_t bytes = o_mask + (size_t)T;
  void* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, bytes);
  if (e != cudaSuccess) return set_error(STORM_ERR_NOMEM, std::string("storm_fvt_link_partitions: ") + cudaGetErrorString(e));
  h->halo_buf = buf;
  char* b = static_cast<char*>(buf);
  if (n_halo > 0) {
    CK(cudaMemcpy(b + o_dst, dst.data(), 4 * (size_t)n_halo, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b + o_src, src.data(), 4 * (size_t)n_halo, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(b + o_mask, mask.data(), (size_t)T, cudaMemcpyHostToDevice));
  h->d.nhalo = n_halo;
  h->d.halo_dst = reinterpret_cast<const int32_t*>(b + o_dst);
  h->d.halo_src = reinterpret_cast<const int32_t*>(b + o_src);
  h->d.halo_mask = reinterpret_cast<const uint8_t*>(b + o_mask);
  h->d.linked = 1;
  h->d.fric_scen = fric_scen;
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->exec = nullptr;
  h->graph = nullptr;
  return capture_graph(h);
}

int storm_fvt_destroy(StormFvtHandle* h) {
  clear_error();
  if (!h) return STORM_OK;
  release(h);
  return STORM_OK;
}

}  // extern "C"
