// Host side of libcps.so: contexts, device memory, launches and the C ABI
// declared in include/cps.h.
//
// Memory: one cudaMalloc'd slab per context.  The ten FP64 field planes (u, v,
// p, p', u*, v*, dE, dN, alpha, gamma) come first, each (M+1) rows x P
// doubles, P = round_up(N+1, 32); then the 25 inner-solve planes in the
// context's storage type (double for CPS_FP64, float for CPS_MIXED); then the
// grid barrier, flags, reduction ring and history buffer.  The fields stay
// resident between calls; per outer iteration only the 8 diagnostics travel
// to the host (batched per call).
//
// Launch, one design: the outer iterations run in one persistent kernel
// launched cooperatively (all CTAs co-resident), synchronised by a software
// grid barrier whose waits are bounded (2 s) and report CPS_ERR_TIMEOUT
// instead of hanging.
//
// Launch, many designs (cps_batch_solve): one thread-block cluster per design
// at a time; clusters take designs from a device work queue, synchronise with
// the hardware cluster barrier and reduce through distributed shared memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/cps.h"
#include "cps_device.cuh"

namespace {

thread_local std::string g_create_error;

constexpr int kHistChunk = 4096;  // outer iterations per launch inside cps_solve
constexpr int kFieldPlanes = 10;  // FP64 planes: u v p pc us vs dE dN alpha gamma
constexpr int kInnerPlanes = 25;  // cU x5, cV x5, bU bV xU0 xU1 xV0 xV1 px pr pz pp0 pp1 pAp pdiag cx cy
constexpr int kMaxGridCtas = 2048;

enum FieldPlane { kU, kV, kP, kPc, kUs, kVs, kDE, kDN, kAlpha, kGamma };

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

struct cps_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int M = 0, N = 0, P = 0;
  int precision = CPS_FP64;
  cps::DesignView view{};
  char* slab = nullptr;
  size_t slab_bytes = 0;
  size_t plane_elems = 0;
  cps::GridBarrier* bar = nullptr;
  double* red = nullptr;
  int* dstatus = nullptr;
  int* dndone = nullptr;
  double* dhist = nullptr;
  double* dplane = nullptr;
  double* hstage = nullptr;  // pinned, one plane of (M+1) x (N+1) doubles
  double* hhist = nullptr;   // pinned, kHistChunk * 8
  int* hflags = nullptr;     // pinned: status, n_done, pressure-drop gate
  double* dplog = nullptr;   // device, kHistChunk x 4 pressure drops of the last launch
  double* hdplog = nullptr;  // pinned copy
  double* ddphist = nullptr; // device, the pressure-drop gate's windows (cudaMalloc'd by cps_set_dp_monitor)
  double* dpseudo = nullptr; // device, the CFL controllers' state (4 doubles)
  cps::TensorMap* dtmaps = nullptr;  // device, the planes' TMA tensor maps (kTmCount), or null
  double pseudo_start = 0.0; // the controllers' starting CFL number
  int ramp_steps = 0;        // inlet velocity ramp of cps_solve (0: off)
  int iter = 0;              // outer-loop iteration index of the next iteration (monitor and gate)
  int grid = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double kernel_ms = 0.0;
  long long launches = 0, outer_done = 0;
  std::string err;
};

// Monitor: the outer loop's pressure-drop monitor and gate compiled in (a
// separate instantiation: compiling it into the plain kernel slowed every
// outer iteration by 60 % on B200).
template <typename T, bool Monitor>
__global__ void __launch_bounds__(cps::kThreads, CPS_MIN_BLOCKS) cps_grid_kernel(cps::DesignView d, cps::RunControl rc,
                                                                cps::GridBarrier* bar, double* red) {
  __shared__ double smem[(Monitor ? cps::kPlaneSums : cps::kRedWidth) * 8];
  __shared__ cps::PseudoRun s_pr;
  extern __shared__ __align__(128) char tile_smem[];
  cps::GridGroup g{bar, red, rc.status, blockIdx.x, gridDim.x, 0u, 0ull};
  if (!cps::tile_buffer_aligned(tile_smem, rc.status)) return;
  cps::tma_barriers_init();
  cps::load_pseudo(d, s_pr);
  __syncthreads();
  cps::SweepHint hint{2, 2, 2};
  for (int it = 0; it < rc.n_outer; ++it) {
    double out[8];
    const int r = cps::outer_iteration<T, cps::GridGroup, Monitor>(
        d, g, smem, tile_smem, out, it + 1 == rc.n_outer, rc.stop_on_conv != 0, rc.eps, rc.iter0 + it,
        rc.dplog ? rc.dplog + (size_t)4 * it : nullptr, rc.dp_converged, &s_pr, &hint);
    if (r < 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      for (int k = 0; k < 8; ++k) rc.hist[(size_t)it * 8 + k] = out[k];
      *rc.n_done = it + 1;
    }
    if (r == 1) return;
  }
}

// Batched solves: each cluster takes the next design from the queue and runs
// its outer iterations to convergence or to the item's budget.
template <typename T, bool Pseudo>
__global__ void __launch_bounds__(cps::kThreads) cps_cluster_kernel(const cps::BatchItem* __restrict__ items,
                                                                   const int* __restrict__ order, int n_items,
                                                                   int* queue, cps::BatchResult* results) {
  __shared__ double smem[cps::kRedWidth * 8];
  __shared__ double redbuf[2 * cps::kRedWidth];
  __shared__ __align__(16) cps::BatchItem s_item;
  __shared__ cps::PseudoRun s_pr;
  __shared__ int s_next;
  extern __shared__ __align__(128) char tile_smem[];
  cps::cg::cluster_group cl = cps::cg::this_cluster();
  cps::ClusterGroup g{redbuf, nullptr, cl.block_rank(), cl.num_blocks(), 0u};
  if (!cps::tile_buffer_aligned(tile_smem, &results[0].status)) return;
  cps::tma_barriers_init();
  for (;;) {
    if (g.rank == 0 && threadIdx.x == 0) s_next = atomicAdd(queue, 1);
    cl.sync();
    const int idx = *cl.map_shared_rank(&s_next, 0);
    if (idx >= n_items) break;
    const int id = order[idx];
    {
      const int* src = reinterpret_cast<const int*>(items + id);
      int* dst = reinterpret_cast<int*>(&s_item);
      for (int k = threadIdx.x; k < (int)(sizeof(cps::BatchItem) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const cps::BatchItem& item = s_item;
    cps::load_pseudo(item.view, s_pr);
    __syncthreads();
    cps::BatchResult* res = results + id;
    g.status = &res->status;
    double out[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int done = 0;
    cps::SweepHint hint{2, 2, 2};
    for (int it = 0; it < item.n_outer; ++it) {
      const int r = cps::outer_iteration<T, cps::ClusterGroup, false, Pseudo>(
          item.view, g, smem, tile_smem, out, it + 1 == item.n_outer, item.stop_on_conv != 0, item.eps, item.iter0 + it,
          nullptr, nullptr, &s_pr, &hint);
      done = it + 1;
      if (g.rank == 0 && threadIdx.x == 0 && item.hist && it < item.hist_cap)
        for (int k = 0; k < 8; ++k) item.hist[(size_t)it * 8 + k] = out[k];
      if (r != 0) break;
    }
    if (g.rank == 0 && threadIdx.x == 0) {
      res->n_done = done;
      const double conv = cps::maxd(cps::maxd(out[0], out[1]), out[3]);
      res->converged = (done > 0 && conv <= item.eps) ? 1 : 0;
      for (int k = 0; k < 8; ++k) res->last[k] = out[k];
    }
    cl.sync();  // s_item, s_next and the reduction ring are reused next round
  }
  cl.sync();    // no CTA leaves while another may still read its shared memory
}

// Batched solves on groups of CTAs inside one cooperative launch: CTAs
// [g*K, (g+1)*K) form group g, which takes designs from the queue one at a
// time and runs each with the bounded software barrier of its own counter.
// The group count sets how many designs are in flight (and so the in-flight
// working set against the 126 MB L2); K sets how many CTAs share one design.
template <typename T, bool Pseudo>
__global__ void __launch_bounds__(cps::kThreads, CPS_MIN_BLOCKS) cps_group_kernel(const cps::BatchItem* __restrict__ items,
                                                                    const int* __restrict__ order, int n_items,
                                                                    int* queue, cps::BatchResult* results,
                                                                    cps::GridBarrier* bars, double* rings,
                                                                    int* slots, int group_ctas) {
  __shared__ double smem[cps::kRedWidth * 8];
  __shared__ __align__(16) cps::BatchItem s_item;
  __shared__ cps::PseudoRun s_pr;
  extern __shared__ __align__(128) char tile_smem[];
  const unsigned grp = blockIdx.x / group_ctas;
  int* slot = slots + 2 * grp;  // [0] next queue index, [1] group status before a design is assigned
  cps::GridGroup g{bars + grp, rings + (size_t)grp * cps::kRedSlots * group_ctas * cps::kRedWidth, slot + 1,
                   blockIdx.x % group_ctas, (unsigned)group_ctas, 0u, 0ull};
  if (!cps::tile_buffer_aligned(tile_smem, &results[0].status)) return;
  cps::tma_barriers_init();
  for (;;) {
    g.status = slot + 1;
    if (g.rank == 0 && threadIdx.x == 0) slot[0] = atomicAdd(queue, 1);
    if (!g.sync()) return;
    const int idx = __ldcg(slot);
    if (!g.sync()) return;  // every CTA has read the index before the leader takes the next one
    if (idx >= n_items) return;
    const int id = order[idx];
    {
      const int* src = reinterpret_cast<const int*>(items + id);
      int* dst = reinterpret_cast<int*>(&s_item);
      for (int k = threadIdx.x; k < (int)(sizeof(cps::BatchItem) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const cps::BatchItem& item = s_item;
    cps::load_pseudo(item.view, s_pr);
    __syncthreads();
    cps::BatchResult* res = results + id;
    g.status = &res->status;
    double out[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int done = 0;
    cps::SweepHint hint{2, 2, 2};
    for (int it = 0; it < item.n_outer; ++it) {
      const int r = cps::outer_iteration<T, cps::GridGroup, false, Pseudo>(
          item.view, g, smem, tile_smem, out, it + 1 == item.n_outer, item.stop_on_conv != 0, item.eps, item.iter0 + it,
          nullptr, nullptr, &s_pr, &hint);
      if (r < 0) return;  // a bounded wait expired; the design's status says so
      done = it + 1;
      if (g.rank == 0 && threadIdx.x == 0 && item.hist && it < item.hist_cap)
        for (int k = 0; k < 8; ++k) item.hist[(size_t)it * 8 + k] = out[k];
      if (r != 0) break;
    }
    if (g.rank == 0 && threadIdx.x == 0) {
      res->n_done = done;
      const double conv = cps::maxd(cps::maxd(out[0], out[1]), out[3]);
      res->converged = (done > 0 && conv <= item.eps) ? 1 : 0;
      for (int k = 0; k < 8; ++k) res->last[k] = out[k];
    }
    __syncthreads();  // s_item is reloaded next round
  }
}

// Batched solves in waves: one design per group, groups sized to their
// designs.  CTAs [first[g], first[g+1]) form group g and run design which[g]
// to convergence or to its budget with the bounded software barrier of their
// own counter; their reduction ring starts at first[g] ring rows.
template <typename T, bool Pseudo>
__global__ void __launch_bounds__(cps::kThreads, CPS_MIN_BLOCKS) cps_wave_kernel(const cps::BatchItem* __restrict__ items,
                                                                   const int* __restrict__ first,
                                                                   const int* __restrict__ which, int groups,
                                                                   cps::BatchResult* results,
                                                                   cps::GridBarrier* bars, double* rings) {
  __shared__ double smem[cps::kRedWidth * 8];
  __shared__ __align__(16) cps::BatchItem s_item;
  __shared__ cps::PseudoRun s_pr;
  extern __shared__ __align__(128) char tile_smem[];
  if (!cps::tile_buffer_aligned(tile_smem, &results[which[0]].status)) return;
  cps::tma_barriers_init();
  int lo = 0, hi = groups;  // first[lo] <= blockIdx.x < first[lo + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= (int)blockIdx.x) lo = mid; else hi = mid;
  }
  const int grp = lo, K = first[grp + 1] - first[grp], id = which[grp];
  {
    const int* src = reinterpret_cast<const int*>(items + id);
    int* dst = reinterpret_cast<int*>(&s_item);
    for (int k = threadIdx.x; k < (int)(sizeof(cps::BatchItem) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
  }
  __syncthreads();
  const cps::BatchItem& item = s_item;
  cps::load_pseudo(item.view, s_pr);
  __syncthreads();
  cps::BatchResult* res = results + id;
  cps::GridGroup g{bars + grp, rings + (size_t)first[grp] * cps::kRedSlots * cps::kRedWidth, &res->status,
                   blockIdx.x - (unsigned)first[grp], (unsigned)K, 0u, 0ull};
  double out[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int done = 0;
  cps::SweepHint hint{2, 2, 2};
  for (int it = 0; it < item.n_outer; ++it) {
    const int r = cps::outer_iteration<T, cps::GridGroup, false, Pseudo>(
        item.view, g, smem, tile_smem, out, it + 1 == item.n_outer, item.stop_on_conv != 0, item.eps, item.iter0 + it,
        nullptr, nullptr, &s_pr, &hint);
    if (r < 0) return;  // a bounded wait expired; the design's status says so
    done = it + 1;
    if (g.rank == 0 && threadIdx.x == 0 && item.hist && it < item.hist_cap)
      for (int k = 0; k < 8; ++k) item.hist[(size_t)it * 8 + k] = out[k];
    if (r != 0) break;
  }
  if (g.rank == 0 && threadIdx.x == 0) {
    res->n_done = done;
    const double conv = cps::maxd(cps::maxd(out[0], out[1]), out[3]);
    res->converged = (done > 0 && conv <= item.eps) ? 1 : 0;
    for (int k = 0; k < 8; ++k) res->last[k] = out[k];
  }
}

// samplePlaneAtX (postprocessing.cpp:62-230) for one plane, one CTA: every row's
// contribution is evaluated with the reference's expressions; the five sums are
// combined in a fixed tree order.
__global__ void __launch_bounds__(cps::kThreads) cps_plane_kernel(cps::DesignView d, double xPhysical, double* out) {
  __shared__ double smem[cps::kRedWidth * 8];
  const cps::PlaneSetup ps = cps::plane_setup(d, xPhysical);
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // staticAreaSum, dynAreaSum, totalWeighted, area, fluxSum
  for (int i = 1 + threadIdx.x; i < d.M; i += blockDim.x) cps::plane_row(d, ps, i, acc);
  cps::block_reduce<5, 0u>(acc, smem);
  if (threadIdx.x == 0) cps::plane_metrics(acc, out);
}

namespace {

bool cuda_ok(cps_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (ctx) ctx->err = m; else g_create_error = m;
  return false;
}

cps_status fail(cps_ctx* ctx, cps_status s, const std::string& msg) {
  if (ctx) ctx->err = msg; else g_create_error = msg;
  return s;
}

size_t elem_bytes(int precision) { return precision == CPS_MIXED ? sizeof(float) : sizeof(double); }

size_t footprint_bytes(int M, int N, int precision, size_t* plane_elems_out, int* P_out) {
  const int P = (int)round_up((size_t)N + 1, 32);
  const size_t plane = (size_t)(M + 1) * P;
  if (plane_elems_out) *plane_elems_out = plane;
  if (P_out) *P_out = P;
  size_t bytes = plane * sizeof(double) * kFieldPlanes;
  bytes += round_up(plane * elem_bytes(precision) * kInnerPlanes, 256);
  bytes += 256;                                                           // barrier + flags
  bytes += (size_t)(cps::kRedSlots * cps::kRedWidth + cps::kPlaneSums) * kMaxGridCtas * 8;  // reduction ring
  bytes += (size_t)kHistChunk * 8 * 8 + 64;                               // history + plane metrics
  bytes += (size_t)kHistChunk * 4 * 8;                                    // pressure-drop log
  bytes += 64;                                                            // CFL controllers' state
  bytes += 128 + sizeof(cps::TensorMap) * cps::kTmCount;                  // TMA tensor maps
  return round_up(bytes, 256);
}

// The CFL controllers' state on the device (pseudoCFL, serResidPrev,
// lsCurrentAlpha, lsBacktrackCount), written in stream order.
bool write_pseudo_state(cps_ctx* c, double cfl, double prev, double alpha, int count) {
  const double h[4] = {cfl, prev, alpha, (double)count};
  return cuda_ok(c, cudaMemcpyAsync(c->dpseudo, h, sizeof(h), cudaMemcpyHostToDevice, c->stream), "h2d") &&
         cuda_ok(c, cudaStreamSynchronize(c->stream), "h2d");
}

// ---------------------------------------------------------------------------
// TMA tensor maps of a context's planes: one 2-D map per (plane, window shape)
// the staged phases copy, over the plane's rows 0..rmax and columns 0..P-1,
// with the window's box (its shared-memory pitch x rows).  Out-of-range parts
// of a box read as zero (the phases never use them).  Built once at
// cps_create and kept in the context's slab.
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

template <typename E, class W>
bool encode_map(PFN_cuTensorMapEncodeTiled_v12000 fn, cps::TensorMap* out, const E* base, int P, int rows) {
  static_assert(sizeof(cps::TensorMap) == sizeof(CUtensorMap), "tensor map size");
  const cuuint64_t dims[2] = {(cuuint64_t)P, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)P * sizeof(E)};
  const cuuint32_t box[2] = {(cuuint32_t)W::kPitch, (cuuint32_t)W::kRows};
  const cuuint32_t estr[2] = {1, 1};
  static_assert(W::kPitch * sizeof(E) % 16 == 0 && W::kPitch <= 256 && W::kRows <= 256, "TMA box");
  return fn(reinterpret_cast<CUtensorMap*>(out), sizeof(E) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
            2, const_cast<E*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T>
bool fill_maps(PFN_cuTensorMapEncodeTiled_v12000 fn, const cps::DesignView& v, const cps::Inner<T>& w, int M, int P,
               cps::TensorMap* m) {
  using LA = cps::LayoutA;
  using LC = cps::LayoutC<T>;
  using LD = cps::LayoutD<T>;
  using LB = cps::LayoutB<T>;
  const int R = M + 1;  // rows 0..M
  const long long ps = v.planeStride;
  for (int q = 0; q < 5; ++q)
    if (!encode_map<T, typename LB::WC>(fn, m + cps::kTmCU_B + q, w.cU + q * ps, P, R) ||
        !encode_map<T, typename LB::WC>(fn, m + cps::kTmCV_B + q, w.cV + q * ps, P, R))
      return false;
  if (!encode_map<T, typename LB::WC>(fn, m + cps::kTmBU_B, w.bU, P, R) ||
      !encode_map<T, typename LB::WC>(fn, m + cps::kTmBV_B, w.bV, P, R) ||
      !encode_map<T, typename LB::WX>(fn, m + cps::kTmXU0_B, w.xU0, P, R) ||
      !encode_map<T, typename LB::WX>(fn, m + cps::kTmXU1_B, w.xU1, P, R) ||
      !encode_map<T, typename LB::WX>(fn, m + cps::kTmXV0_B, w.xV0, P, R) ||
      !encode_map<T, typename LB::WX>(fn, m + cps::kTmXV1_B, w.xV1, P, R))
    return false;
  return encode_map<double, LA::WU>(fn, m + cps::kTmU_A, v.u, P, R) &&
         encode_map<double, LA::WU>(fn, m + cps::kTmV_A, v.v, P, R) &&
         encode_map<double, LA::WP>(fn, m + cps::kTmP_A, v.p, P, R) &&
         encode_map<double, LA::WA>(fn, m + cps::kTmAlpha_A, v.alpha, P, M) &&
         encode_map<T, typename LC::WUx>(fn, m + cps::kTmXU0_C, w.xU0, P, R) &&
         encode_map<T, typename LC::WUx>(fn, m + cps::kTmXU1_C, w.xU1, P, R) &&
         encode_map<double, typename LC::WUd>(fn, m + cps::kTmU_C, v.u, P, R) &&
         encode_map<double, typename LC::WUd>(fn, m + cps::kTmDE_C, v.dE, P, R) &&
         encode_map<T, typename LC::WVx>(fn, m + cps::kTmXV0_C, w.xV0, P, R) &&
         encode_map<T, typename LC::WVx>(fn, m + cps::kTmXV1_C, w.xV1, P, R) &&
         encode_map<double, typename LC::WVd>(fn, m + cps::kTmV_C, v.v, P, R) &&
         encode_map<double, typename LC::WVd>(fn, m + cps::kTmDN_C, v.dN, P, R) &&
         encode_map<double, typename LC::WG>(fn, m + cps::kTmG_C, v.gamma, P, M) &&
         encode_map<T, typename LD::WX>(fn, m + cps::kTmPX_D, w.px, P, R) &&
         encode_map<double, typename LD::WO>(fn, m + cps::kTmP_D, v.p, P, R) &&
         encode_map<double, typename LD::WO>(fn, m + cps::kTmDE_D, v.dE, P, R) &&
         encode_map<double, typename LD::WO>(fn, m + cps::kTmUS_D, v.us, P, R) &&
         encode_map<double, typename LD::WO>(fn, m + cps::kTmDN_D, v.dN, P, R) &&
         encode_map<double, typename LD::WO>(fn, m + cps::kTmVS_D, v.vs, P, R) &&
         encode_map<double, typename LD::WG>(fn, m + cps::kTmG_D, v.gamma, P, M);
}

// The context's tensor maps, or false (the staged phases then copy element by
// element): no driver entry point, an encoding refused, or CPS_STAGING=elements
// in the environment (the element-wise path, for comparisons).
bool build_tensor_maps(cps_ctx* c) {
  const char* mode = std::getenv("CPS_STAGING");
  if (mode && std::strcmp(mode, "elements") == 0) return false;
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_tiled();
  if (!fn) return false;
  cps::TensorMap h[cps::kTmCount];
  std::memset(h, 0, sizeof(h));
  const bool ok = c->precision == CPS_MIXED ? fill_maps<float>(fn, c->view, c->view.f32, c->M, c->P, h)
                                            : fill_maps<double>(fn, c->view, c->view.f64, c->M, c->P, h);
  if (!ok) return false;
  return cudaMemcpyAsync(c->dtmaps, h, sizeof(h), cudaMemcpyHostToDevice, c->stream) == cudaSuccess &&
         cudaStreamSynchronize(c->stream) == cudaSuccess;
}

cps_status validate(const cps_desc* d) {
  if (!d) return fail(nullptr, CPS_ERR_ARG, "desc is NULL");
  if (d->M < 3 || d->N < 3) return fail(nullptr, CPS_ERR_ARG, "grid too small: need M >= 3 and N >= 3");
  if ((long long)d->M * d->N > (1LL << 28)) return fail(nullptr, CPS_ERR_ARG, "grid too large");
  if (!(d->hx > 0) || !(d->hy > 0) || !(d->rho > 0) || !(d->eta > 0))
    return fail(nullptr, CPS_ERR_ARG, "hx, hy, rho and eta must be positive");
  if (!(d->uvAlpha > 0) || !(d->pAlpha >= 0)) return fail(nullptr, CPS_ERR_ARG, "bad relaxation factors");
  if (d->maxPressureIter < 0 || d->maxMomentumIter < 0) return fail(nullptr, CPS_ERR_ARG, "negative iteration cap");
  if (d->precision != CPS_FP64 && d->precision != CPS_MIXED) return fail(nullptr, CPS_ERR_ARG, "bad precision");
  if (d->layout != CPS_ROW_MAJOR && d->layout != CPS_COL_MAJOR) return fail(nullptr, CPS_ERR_ARG, "bad layout");
  if (!d->alpha || !d->gamma) return fail(nullptr, CPS_ERR_ARG, "alpha and gamma are required");
  if (d->grid_ctas < 0) return fail(nullptr, CPS_ERR_ARG, "grid_ctas < 0");
  if (d->pcg_variant != CPS_PCG_REFERENCE && d->pcg_variant != CPS_PCG_SINGLE_REDUCTION)
    return fail(nullptr, CPS_ERR_ARG, "bad pcg_variant");
  if (d->momentum_explicit != 0 && d->momentum_explicit != 1)
    return fail(nullptr, CPS_ERR_ARG, "momentum_explicit must be 0 (implicit Jacobi) or 1 (explicit)");
  return CPS_OK;
}

// Copy a host rows x cols matrix (row- or column-major) into a pitched device plane.
bool upload_plane(cps_ctx* c, double* dst, const double* src, int rows, int cols, int layout) {
  if (layout == CPS_COL_MAJOR) {
    for (int i = 0; i < rows; ++i)
      for (int j = 0; j < cols; ++j) c->hstage[(size_t)i * cols + j] = src[(size_t)j * rows + i];
  } else {
    std::memcpy(c->hstage, src, sizeof(double) * (size_t)rows * cols);
  }
  if (!cuda_ok(c, cudaMemcpy2DAsync(dst, (size_t)c->P * 8, c->hstage, (size_t)cols * 8, (size_t)cols * 8, rows,
                                    cudaMemcpyHostToDevice, c->stream), "upload"))
    return false;
  return cuda_ok(c, cudaStreamSynchronize(c->stream), "upload sync");
}

bool download_plane(cps_ctx* c, double* dst, const double* src, int rows, int cols, int layout) {
  if (!dst) return true;
  if (!cuda_ok(c, cudaMemcpy2DAsync(c->hstage, (size_t)cols * 8, src, (size_t)c->P * 8, (size_t)cols * 8, rows,
                                    cudaMemcpyDeviceToHost, c->stream), "download"))
    return false;
  if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "download sync")) return false;
  if (layout == CPS_COL_MAJOR) {
    for (int i = 0; i < rows; ++i)
      for (int j = 0; j < cols; ++j) dst[(size_t)j * rows + i] = c->hstage[(size_t)i * cols + j];
  } else {
    std::memcpy(dst, c->hstage, sizeof(double) * (size_t)rows * cols);
  }
  return true;
}

double* field_ptr(cps_ctx* c, int k) { return reinterpret_cast<double*>(c->slab) + (size_t)k * c->plane_elems; }

template <typename T>
void bind_inner(cps_ctx* c, cps::Inner<T>& w) {
  T* base = reinterpret_cast<T*>(c->slab + c->plane_elems * sizeof(double) * kFieldPlanes);
  auto pl = [&](int k) { return base + (size_t)k * c->plane_elems; };
  w.cU = pl(0); w.cV = pl(5);
  w.bU = pl(10); w.bV = pl(11);
  w.xU0 = pl(12); w.xU1 = pl(13); w.xV0 = pl(14); w.xV1 = pl(15);
  w.px = pl(16); w.pr = pl(17); w.pz = pl(18); w.pp0 = pl(19); w.pp1 = pl(20); w.pAp = pl(21);
  w.pdiag = pl(22); w.cx = pl(23); w.cy = pl(24);
}

void set_step_inputs(cps_ctx* c, double Uin) {
  c->view.Uin = Uin;
  c->view.maxVel = 3.0 * std::max(std::fabs(Uin), 0.1);  // iterations.cpp:104
}

const void* grid_kernel_for(int precision, bool monitor = false) {
  if (monitor)
    return precision == CPS_MIXED ? (const void*)cps_grid_kernel<float, true> : (const void*)cps_grid_kernel<double, true>;
  return precision == CPS_MIXED ? (const void*)cps_grid_kernel<float, false> : (const void*)cps_grid_kernel<double, false>;
}

// Dynamic shared memory of the persistent kernels (tile staging buffers).
size_t tile_smem_for(int precision) {
  return precision == CPS_MIXED ? cps::tile_smem_bytes<float>() : cps::tile_smem_bytes<double>();
}

// Let kernel fn use `bytes` of dynamic shared memory on the current device.
bool allow_smem(cps_ctx* c, const void* fn, size_t bytes) {
  return cuda_ok(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), "smem attribute");
}

void to_step_out(const double* h, cps_step_out* o) {
  o->residU = h[0]; o->residV = h[1]; o->residMass = h[2]; o->residMassDof = h[3]; o->err = h[4];
  o->pIters = (int)h[5]; o->uSweeps = (int)h[6]; o->vSweeps = (int)h[7];
}

cps_status run(cps_ctx* c, int n_outer, int stop_on_conv, double eps, cps_step_out* hist, int* n_done,
               double* dp_history = nullptr, int* dp_converged = nullptr, bool ramp = false) {
  int done_total = 0;
  const bool monitor = c->view.dpMonitor != 0;
  const double target = c->view.Uin;
  if (dp_converged) *dp_converged = 0;
  while (done_total < n_outer) {
    int chunk = std::min(kHistChunk, n_outer - done_total);
    if (ramp && c->ramp_steps > 0) {
      // SIMPLE.cpp:303-307: one launch per ramp iteration, each with its own inlet velocity
      if (c->iter < c->ramp_steps) {
        chunk = 1;
        set_step_inputs(c, ((double)(c->iter + 1) / c->ramp_steps) * target);
      } else {
        set_step_inputs(c, target);
      }
    }
    cps::RunControl rc{chunk, stop_on_conv, eps, c->dhist, c->dndone, c->dstatus, c->iter,
                       monitor ? c->dplog : nullptr, c->dstatus + 2};
    if (!cuda_ok(c, cudaMemsetAsync(c->dndone, 0, 2 * sizeof(int), c->stream), "memset") ||
        !cuda_ok(c, cudaMemsetAsync(c->bar, 0, sizeof(cps::GridBarrier), c->stream), "memset"))
      return CPS_ERR_CUDA;
    void* args[] = {&c->view, &rc, &c->bar, &c->red};
    if (!cuda_ok(c, cudaEventRecord(c->ev0, c->stream), "event")) return CPS_ERR_CUDA;
    if (!cuda_ok(c, cudaLaunchCooperativeKernel(grid_kernel_for(c->precision, monitor), dim3(c->grid), dim3(cps::kThreads),
                                                args, tile_smem_for(c->precision), c->stream), "cooperative launch"))
      return CPS_ERR_CUDA;
    if (!cuda_ok(c, cudaEventRecord(c->ev1, c->stream), "event")) return CPS_ERR_CUDA;
    if (!cuda_ok(c, cudaMemcpyAsync(c->hflags, c->dstatus, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->stream), "d2h"))
      return CPS_ERR_CUDA;
    if (monitor && dp_history &&
        !cuda_ok(c, cudaMemcpyAsync(c->hdplog, c->dplog, sizeof(double) * 4 * chunk, cudaMemcpyDeviceToHost,
                                    c->stream), "d2h"))
      return CPS_ERR_CUDA;
    if (!cuda_ok(c, cudaMemcpyAsync(c->hhist, c->dhist, sizeof(double) * 8 * chunk, cudaMemcpyDeviceToHost, c->stream),
                 "d2h"))
      return CPS_ERR_CUDA;
    if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "kernel")) return CPS_ERR_CUDA;
    const int status = c->hflags[0], nd = c->hflags[1];
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, c->ev0, c->ev1) == cudaSuccess) c->kernel_ms += ms;
    c->launches += 1;
    c->outer_done += nd;
    if (hist)
      for (int k = 0; k < nd; ++k) to_step_out(c->hhist + (size_t)8 * k, &hist[done_total + k]);
    if (monitor && dp_history) std::memcpy(dp_history + (size_t)4 * done_total, c->hdplog, sizeof(double) * 4 * nd);
    if (dp_converged && c->hflags[2]) *dp_converged = 1;
    c->iter += nd;
    done_total += nd;
    if (n_done) *n_done = done_total;
    if (status != cps::kStatusOk) {
      // Reset the barrier and status so the context stays usable.
      cudaMemsetAsync(c->bar, 0, sizeof(cps::GridBarrier), c->stream);
      cudaMemsetAsync(c->dstatus, 0, sizeof(int), c->stream);
      cudaStreamSynchronize(c->stream);
      if (status == cps::kStatusTimeout) return fail(c, CPS_ERR_TIMEOUT, "device grid barrier timed out");
      return fail(c, CPS_ERR_DIVERGED, "residual is not finite (solution diverged)");
    }
    if (nd < chunk) break;  // converged
  }
  if (ramp && c->ramp_steps > 0) set_step_inputs(c, target);
  return CPS_OK;
}

// Per-device scratch of cps_batch_solve, grown on demand and reused.
struct BatchWorkspace {
  int device = -1;
  size_t cap = 0;
  cps::BatchItem* items = nullptr;
  int* order = nullptr;
  int* queue = nullptr;
  cps::BatchResult* results = nullptr;
  cps::BatchItem* h_items = nullptr;
  int* h_order = nullptr;
  cps::BatchResult* h_results = nullptr;
  cps::GridBarrier* bars = nullptr;  // group kernel: one barrier, ring and slot pair per group
  double* rings = nullptr;
  int* slots = nullptr;
  int* plan = nullptr;    // wave kernel: per wave, first[groups + 1] then which[groups]
  int* h_plan = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};
std::mutex g_batch_mutex;
std::vector<BatchWorkspace> g_batch_ws;

BatchWorkspace* batch_workspace(int device, size_t n, std::string& err) {
  BatchWorkspace* ws = nullptr;
  for (auto& w : g_batch_ws)
    if (w.device == device) ws = &w;
  if (!ws) {
    g_batch_ws.emplace_back();
    ws = &g_batch_ws.back();
    ws->device = device;
    if (cudaEventCreate(&ws->ev0) != cudaSuccess || cudaEventCreate(&ws->ev1) != cudaSuccess ||
        cudaMalloc(&ws->bars, sizeof(cps::GridBarrier) * kMaxGridCtas) != cudaSuccess ||
        cudaMalloc(&ws->rings, sizeof(double) * cps::kRedSlots * kMaxGridCtas * cps::kRedWidth) != cudaSuccess ||
        cudaMalloc(&ws->slots, sizeof(int) * 2 * kMaxGridCtas) != cudaSuccess) {
      err = "batch workspace allocation failed";
      return nullptr;
    }
  }
  if (ws->cap < n) {
    cudaFree(ws->items); cudaFree(ws->order); cudaFree(ws->queue); cudaFree(ws->results); cudaFree(ws->plan);
    cudaFreeHost(ws->h_items); cudaFreeHost(ws->h_order); cudaFreeHost(ws->h_results); cudaFreeHost(ws->h_plan);
    ws->items = nullptr; ws->order = nullptr; ws->queue = nullptr; ws->results = nullptr; ws->plan = nullptr;
    ws->h_items = nullptr; ws->h_order = nullptr; ws->h_results = nullptr; ws->h_plan = nullptr;
    ws->cap = 0;
    const size_t cap = std::max<size_t>(n, 64);
    if (cudaMalloc(&ws->items, cap * sizeof(cps::BatchItem)) != cudaSuccess ||
        cudaMalloc(&ws->order, cap * sizeof(int)) != cudaSuccess || cudaMalloc(&ws->queue, 256) != cudaSuccess ||
        cudaMalloc(&ws->results, cap * sizeof(cps::BatchResult)) != cudaSuccess ||
        cudaMalloc(&ws->plan, 3 * cap * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&ws->h_plan, 3 * cap * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&ws->h_items, cap * sizeof(cps::BatchItem)) != cudaSuccess ||
        cudaMallocHost(&ws->h_order, cap * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&ws->h_results, cap * sizeof(cps::BatchResult)) != cudaSuccess) {
      err = "batch workspace allocation failed";
      return nullptr;
    }
    ws->cap = cap;
  }
  return ws;
}

}  // namespace

// The persistent kernels' grid barrier, told to expect `expect` CTAs: with more
// than the launch has, the count it waits for is never reached and the wait
// ends only by its time limit (cps_barrier_selftest).
__global__ void __launch_bounds__(cps::kThreads) cps_barrier_selftest_kernel(cps::GridBarrier* bar, int* status,
                                                                            unsigned expect) {
  cps::GridGroup g{bar, nullptr, status, blockIdx.x, expect, 0u, 0ull};
  g.sync();
}

extern "C" {

const char* cps_version(void) { return "cps 0.2 (sm_100a)"; }

cps_status cps_tile_shape(int* rows, int* cols) {
  if (!rows || !cols) return fail(nullptr, CPS_ERR_ARG, "null output");
  *rows = cps::kTileI;
  *cols = cps::kTileJ;
  return CPS_OK;
}

const char* cps_last_error(const cps_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

cps_status cps_barrier_selftest(int device, int ctas, double* kernel_ms) {
  if (ctas < 1 || ctas > 1024) return fail(nullptr, CPS_ERR_ARG, "ctas must be in 1..1024");
  if (kernel_ms) *kernel_ms = 0.0;
  if (!cuda_ok(nullptr, cudaSetDevice(device), "cudaSetDevice")) return CPS_ERR_CUDA;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  char* mem = nullptr;
  int status = -1;
  float ms = 0.0f;
  // counter at [0], status at [64]
  bool ok = cuda_ok(nullptr, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream") &&
            cuda_ok(nullptr, cudaMalloc(&mem, 128), "device allocation") &&
            cuda_ok(nullptr, cudaEventCreate(&e0), "event") && cuda_ok(nullptr, cudaEventCreate(&e1), "event") &&
            cuda_ok(nullptr, cudaMemsetAsync(mem, 0, 128, st), "memset") &&
            cuda_ok(nullptr, cudaEventRecord(e0, st), "event");
  if (ok) {
    cps_barrier_selftest_kernel<<<ctas, cps::kThreads, 0, st>>>(reinterpret_cast<cps::GridBarrier*>(mem),
                                                                 reinterpret_cast<int*>(mem + 64), (unsigned)ctas + 1u);
    ok = cuda_ok(nullptr, cudaGetLastError(), "launch") && cuda_ok(nullptr, cudaEventRecord(e1, st), "event") &&
         cuda_ok(nullptr, cudaMemcpyAsync(&status, mem + 64, sizeof(int), cudaMemcpyDeviceToHost, st), "d2h") &&
         cuda_ok(nullptr, cudaStreamSynchronize(st), "barrier self-test") &&
         cuda_ok(nullptr, cudaEventElapsedTime(&ms, e0, e1), "event time");
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (mem) cudaFree(mem);
  if (st) cudaStreamDestroy(st);
  if (!ok) return CPS_ERR_CUDA;
  if (kernel_ms) *kernel_ms = ms;
  if (status == cps::kStatusTimeout) return fail(nullptr, CPS_ERR_TIMEOUT, "device grid barrier timed out");
  if (status == cps::kStatusOk) return CPS_OK;
  return fail(nullptr, CPS_ERR_STATE, "barrier self-test: unexpected device status");
}

cps_status cps_footprint(const cps_desc* desc, unsigned long long* bytes) {
  cps_status s = validate(desc);
  if (s != CPS_OK) return s;
  if (!bytes) return fail(nullptr, CPS_ERR_ARG, "bytes is NULL");
  *bytes = footprint_bytes(desc->M, desc->N, desc->precision, nullptr, nullptr);
  return CPS_OK;
}

cps_status cps_create(const cps_desc* d, cps_ctx** out) {
  if (!out) return fail(nullptr, CPS_ERR_ARG, "out is NULL");
  *out = nullptr;
  cps_status s = validate(d);
  if (s != CPS_OK) return s;
  cps_ctx* c = new (std::nothrow) cps_ctx();
  if (!c) return fail(nullptr, CPS_ERR_OOM, "host allocation failed");
  c->device = d->device;
  c->M = d->M;
  c->N = d->N;
  c->precision = d->precision;
  c->slab_bytes = footprint_bytes(d->M, d->N, d->precision, &c->plane_elems, &c->P);
  auto bail = [&](cps_status st) {
    g_create_error = c->err;
    cps_destroy(c);
    return st;
  };
  if (!cuda_ok(c, cudaSetDevice(d->device), "cudaSetDevice")) return bail(CPS_ERR_CUDA);
  if (!cuda_ok(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")) return bail(CPS_ERR_CUDA);
  cudaError_t e = cudaMalloc(&c->slab, c->slab_bytes);
  if (e != cudaSuccess) {
    cuda_ok(c, e, "cudaMalloc");
    return bail(CPS_ERR_OOM);
  }
  if (!cuda_ok(c, cudaMemsetAsync(c->slab, 0, c->slab_bytes, c->stream), "memset")) return bail(CPS_ERR_CUDA);
  if (!cuda_ok(c, cudaEventCreate(&c->ev0), "event") || !cuda_ok(c, cudaEventCreate(&c->ev1), "event"))
    return bail(CPS_ERR_CUDA);
  const size_t stage = (size_t)(d->M + 1) * (d->N + 1);
  if (!cuda_ok(c, cudaMallocHost(&c->hstage, stage * sizeof(double)), "pinned alloc") ||
      !cuda_ok(c, cudaMallocHost(&c->hhist, (size_t)kHistChunk * 8 * sizeof(double)), "pinned alloc") ||
      !cuda_ok(c, cudaMallocHost(&c->hflags, 4 * sizeof(int)), "pinned alloc") ||
      !cuda_ok(c, cudaMallocHost(&c->hdplog, sizeof(double) * 4 * kHistChunk), "pinned alloc"))
    return bail(CPS_ERR_OOM);

  char* tail = c->slab + c->plane_elems * sizeof(double) * kFieldPlanes +
               round_up(c->plane_elems * elem_bytes(d->precision) * kInnerPlanes, 256);
  c->bar = reinterpret_cast<cps::GridBarrier*>(tail);
  c->dstatus = reinterpret_cast<int*>(tail + 64);  // [0] status, [1] n_done
  c->dndone = c->dstatus + 1;
  c->red = reinterpret_cast<double*>(tail + 256);
  c->dhist = c->red + (size_t)(cps::kRedSlots * cps::kRedWidth + cps::kPlaneSums) * kMaxGridCtas;
  c->dplane = c->dhist + (size_t)kHistChunk * 8;
  c->dplog = c->dplane + 8;
  c->dpseudo = c->dplog + (size_t)4 * kHistChunk;
  c->dtmaps = reinterpret_cast<cps::TensorMap*>(round_up(reinterpret_cast<size_t>(c->dpseudo + 8), 128));

  cps::DesignView& v = c->view;
  v.M = d->M; v.N = d->N; v.P = c->P;
  v.conv = d->convectionScheme; v.maxPIter = d->maxPressureIter; v.maxMomIter = d->maxMomentumIter;
  v.pcgSingleReduction = d->pcg_variant == CPS_PCG_SINGLE_REDUCTION ? 1 : 0;
  v.momExplicit = d->momentum_explicit;
  v.hx = d->hx; v.hy = d->hy; v.rho = d->rho; v.uvAlpha = d->uvAlpha; v.pAlpha = d->pAlpha; v.pTol = d->pTol;
  // Derived constants, evaluated in the reference's operation order
  // (momentum_solver.cpp:166-191, 220-222, 261; jacobi_solver.cpp:41, 63).
  v.vol = d->hx * d->hy;
  v.De = d->eta * d->hy / d->hx;
  v.Dn = d->eta * d->hx / d->hy;
  const double sinkCoeff = (d->enableTwoPointFiveD && d->Ht_channel > 0.0)
                               ? d->twoPointFiveDSinkMultiplier * (5.0 * d->eta / (2.0 * d->Ht_channel * d->Ht_channel))
                               : 0.0;
  v.sinkDiag = sinkCoeff * v.vol;
  const double convScale = d->enableConvectionScaling ? (6.0 / 7.0) : 1.0;
  v.Fcx = convScale * d->rho * d->hy;
  v.Fcy = convScale * d->rho * d->hx;
  v.relax = (1.0 - d->uvAlpha) / d->uvAlpha;
  const double tolsq = d->momentumTol * d->momentumTol;
  v.thrU = tolsq * (double)((d->M - 1) * (d->N - 2));
  v.thrV = tolsq * (double)((d->M - 2) * (d->N - 1));
  v.u = field_ptr(c, kU); v.v = field_ptr(c, kV); v.p = field_ptr(c, kP); v.pc = field_ptr(c, kPc);
  v.us = field_ptr(c, kUs); v.vs = field_ptr(c, kVs); v.dE = field_ptr(c, kDE); v.dN = field_ptr(c, kDN);
  v.alpha = field_ptr(c, kAlpha); v.gamma = field_ptr(c, kGamma);
  v.planeStride = (long long)c->plane_elems;
  std::memset(&v.f64, 0, sizeof(v.f64));
  std::memset(&v.f32, 0, sizeof(v.f32));
  if (d->precision == CPS_MIXED) bind_inner<float>(c, v.f32); else bind_inner<double>(c, v.f64);
  set_step_inputs(c, 0.0);
  v.tm = build_tensor_maps(c) ? c->dtmaps : nullptr;
  {
    // The Jacobi sweeps load straight from global memory: staging their tiles
    // by TMA gave the same bits but measured 0-1.5 % slower per outer
    // iteration (the sweeps are not bound by their loads' latency).
    // CPS_STAGE_SWEEPS=1 in the environment stages them (for comparisons).
    const char* sw = std::getenv("CPS_STAGE_SWEEPS");
    v.stageSweeps = (sw && std::strcmp(sw, "1") == 0) ? 1 : 0;
  }

  if (!upload_plane(c, v.alpha, d->alpha, d->M, d->N, d->layout) ||
      !upload_plane(c, v.gamma, d->gamma, d->M, d->N, d->layout))
    return bail(CPS_ERR_CUDA);

  // Persistent grid: co-resident CTAs, at most one per tile of the design.
  int per_sm = 0, sms = 0;
  if (!allow_smem(c, grid_kernel_for(d->precision), tile_smem_for(d->precision)) ||
      !allow_smem(c, grid_kernel_for(d->precision, true), tile_smem_for(d->precision)) ||
      !cuda_ok(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_kernel_for(d->precision),
                                                                cps::kThreads, tile_smem_for(d->precision)),
               "occupancy") ||
      !cuda_ok(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device), "attribute"))
    return bail(CPS_ERR_CUDA);
  if (per_sm < 1) return bail(fail(c, CPS_ERR_CUDA, "persistent kernel does not fit on an SM"));
  const int tiles = ((d->M - 1 + cps::kTileI - 1) / cps::kTileI) * ((d->N - 1 + cps::kTileJ - 1) / cps::kTileJ);
  // Default: the fewest rounds of tiles per CTA the co-resident CTAs allow,
  // with the tiles spread evenly (every CTA takes part in every barrier).
  const int cap = std::min(sms * per_sm, kMaxGridCtas);
  const int rounds = (tiles + cap - 1) / cap;
  int grid = d->grid_ctas > 0 ? d->grid_ctas : (tiles + rounds - 1) / rounds;
  grid = std::min(grid, cap);
  grid = std::max(1, std::min(grid, tiles));
  c->grid = grid;
  *out = c;
  return CPS_OK;
}

void cps_destroy(cps_ctx* c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->slab) cudaFree(c->slab);
  if (c->hstage) cudaFreeHost(c->hstage);
  if (c->hhist) cudaFreeHost(c->hhist);
  if (c->hflags) cudaFreeHost(c->hflags);
  if (c->hdplog) cudaFreeHost(c->hdplog);
  if (c->ddphist) cudaFree(c->ddphist);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

cps_status cps_upload_geometry(cps_ctx* c, const double* alpha, const double* gamma, int layout) {
  if (!c || !alpha || !gamma) return fail(c, CPS_ERR_ARG, "ctx, alpha and gamma are required");
  if (layout != CPS_ROW_MAJOR && layout != CPS_COL_MAJOR) return fail(c, CPS_ERR_ARG, "bad layout");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  if (!upload_plane(c, c->view.alpha, alpha, c->M, c->N, layout) ||
      !upload_plane(c, c->view.gamma, gamma, c->M, c->N, layout))
    return CPS_ERR_CUDA;
  return CPS_OK;
}

cps_status cps_reset_fields(cps_ctx* c) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  // Planes u .. dN are contiguous at the start of the slab.
  if (!cuda_ok(c, cudaMemsetAsync(c->slab, 0, c->plane_elems * sizeof(double) * (kDN + 1), c->stream), "memset"))
    return CPS_ERR_CUDA;
  c->iter = 0;
  if (c->view.pseudo && !write_pseudo_state(c, c->pseudo_start, 0.0, 1.0, 0)) return CPS_ERR_CUDA;
  return CPS_OK;
}

cps_status cps_pseudo_defaults(cps_pseudo* p, double target_velocity) {
  if (!p) return fail(nullptr, CPS_ERR_ARG, "p is NULL");
  cps_pseudo q;
  std::memset(&q, 0, sizeof(q));
  // SIMPLE.h:255-313
  q.enable = 0;
  q.use_local = 1;
  q.enable_ser = 1;
  q.enable_line_search = 1;
  q.enable_cfl_ramp = 1;
  q.ser_use_max_resid = 0;
  q.ser_min_iter = 10;
  q.ls_max_tries = 4;
  q.target_velocity = target_velocity;
  q.time_step_multiplier = 0.01;
  q.min_pseudo_speed = 0.05;
  q.pseudo_cfl = 0.1;
  q.cfl_initial = 0.1;
  q.cfl_max = 30.0;
  q.cfl_ramp_start_res = 1e-4;
  q.cfl_ramp_exponent = 0.8;
  q.cfl_ramp_smooth = 0.1;
  q.ser_cfl_min = 0.1;
  q.ser_cfl_max = 5.0;
  q.ser_smooth = 0.5;
  q.ser_max_increase = 1.1;
  q.ser_max_decrease = 0.7;
  q.ls_alpha_min = 0.1;
  q.ls_alpha_reduce = 0.3;
  q.ls_resid_increase_tol = 1.01;
  *p = q;
  return CPS_OK;
}

cps_status cps_set_pseudo(cps_ctx* c, const cps_pseudo* p) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  cps::DesignView& v = c->view;
  if (!p || !p->enable) {
    v.pseudo = 0;
    return CPS_OK;
  }
  const double reals[] = {p->time_step, p->target_velocity, p->time_step_multiplier, p->min_pseudo_speed, p->pseudo_cfl,
                          p->cfl_initial, p->cfl_max, p->cfl_ramp_start_res, p->cfl_ramp_exponent,
                          p->cfl_ramp_smooth, p->ser_cfl_min, p->ser_cfl_max, p->ser_smooth, p->ser_max_increase,
                          p->ser_max_decrease, p->ls_alpha_min, p->ls_alpha_reduce, p->ls_resid_increase_tol};
  for (double x : reals)
    if (!std::isfinite(x)) return fail(c, CPS_ERR_ARG, "pseudo-transient parameters must be finite");
  if (!(p->time_step_multiplier > 0.0 || p->time_step > 0.0) || p->ser_min_iter < 0 || p->ls_max_tries < 0)
    return fail(c, CPS_ERR_ARG,
                "pseudo-transient: time_step or time_step_multiplier > 0, ser_min_iter >= 0, ls_max_tries >= 0");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  v.pseudoLocal = p->use_local ? 1 : 0;
  v.serOn = p->enable_ser ? 1 : 0;
  v.lsOn = p->enable_line_search ? 1 : 0;
  v.rampOn = p->enable_cfl_ramp ? 1 : 0;
  v.serUseMax = p->ser_use_max_resid ? 1 : 0;
  v.serMinIter = p->ser_min_iter;
  v.lsMaxTries = p->ls_max_tries;
  // SIMPLE.cpp:68-70, in the reference's operation order
  const double domainLength = c->N * v.hx;
  const double velRef = std::max(p->target_velocity, 1e-6);
  v.timeStep = p->time_step > 0.0 ? p->time_step : p->time_step_multiplier * domainLength / velRef;
  v.minPseudoSpeed = p->min_pseudo_speed;
  v.hChar = std::min(v.hx, v.hy);  // momentum_solver.cpp:190, iterations.cpp:189
  v.cflInitial = p->cfl_initial;
  v.cflMax = p->cfl_max;
  v.rampStartRes = p->cfl_ramp_start_res;
  v.rampExponent = p->cfl_ramp_exponent;
  v.rampSmooth = p->cfl_ramp_smooth;
  v.serCFLMin = p->ser_cfl_min;
  v.serCFLMax = p->ser_cfl_max;
  v.serSmooth = p->ser_smooth;
  v.serMaxIncrease = p->ser_max_increase;
  v.serMaxDecrease = p->ser_max_decrease;
  v.lsAlphaMin = p->ls_alpha_min;
  v.lsAlphaReduce = p->ls_alpha_reduce;
  v.lsTol = p->ls_resid_increase_tol;
  v.pseudoState = c->dpseudo;
  // the constructor starts the ramp at pseudoCFLInitial (SIMPLE.cpp:78-82)
  c->pseudo_start = p->enable_cfl_ramp ? p->cfl_initial : p->pseudo_cfl;
  if (!write_pseudo_state(c, c->pseudo_start, 0.0, 1.0, 0)) return CPS_ERR_CUDA;
  v.pseudo = 1;
  return CPS_OK;
}

cps_status cps_get_pseudo_state(cps_ctx* c, cps_pseudo_state* state) {
  if (!c || !state) return fail(c, CPS_ERR_ARG, "ctx and state are required");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  double h[4];
  if (!cuda_ok(c, cudaMemcpyAsync(h, c->dpseudo, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "d2h") ||
      !cuda_ok(c, cudaStreamSynchronize(c->stream), "d2h"))
    return CPS_ERR_CUDA;
  state->pseudo_cfl = h[0];
  state->ser_resid_prev = h[1];
  state->ls_alpha = h[2];
  state->ls_backtracks = (int)h[3];
  state->pad = 0;
  return CPS_OK;
}

cps_status cps_set_pseudo_state(cps_ctx* c, const cps_pseudo_state* state) {
  if (!c || !state) return fail(c, CPS_ERR_ARG, "ctx and state are required");
  if (!std::isfinite(state->pseudo_cfl) || !std::isfinite(state->ser_resid_prev) || !std::isfinite(state->ls_alpha))
    return fail(c, CPS_ERR_ARG, "pseudo state must be finite");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  return write_pseudo_state(c, state->pseudo_cfl, state->ser_resid_prev, state->ls_alpha, state->ls_backtracks)
             ? CPS_OK
             : CPS_ERR_CUDA;
}

cps_status cps_get_stream(cps_ctx* c, void** stream) {
  if (!c || !stream) return fail(c, CPS_ERR_ARG, "ctx and stream are required");
  *stream = (void*)c->stream;
  return CPS_OK;
}

cps_status cps_kernel_timing(cps_ctx* c, double* kernel_ms, long long* launches, long long* outer_iterations,
                             int reset) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (kernel_ms) *kernel_ms = c->kernel_ms;
  if (launches) *launches = c->launches;
  if (outer_iterations) *outer_iterations = c->outer_done;
  if (reset) { c->kernel_ms = 0.0; c->launches = 0; c->outer_done = 0; }
  return CPS_OK;
}

cps_status cps_upload_fields(cps_ctx* c, const double* u, const double* v, const double* p, int layout) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (layout != CPS_ROW_MAJOR && layout != CPS_COL_MAJOR) return fail(c, CPS_ERR_ARG, "bad layout");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  if (u && !upload_plane(c, c->view.u, u, c->M + 1, c->N, layout)) return CPS_ERR_CUDA;
  if (v && !upload_plane(c, c->view.v, v, c->M, c->N + 1, layout)) return CPS_ERR_CUDA;
  if (p && !upload_plane(c, c->view.p, p, c->M + 1, c->N + 1, layout)) return CPS_ERR_CUDA;
  return CPS_OK;
}

cps_status cps_step(cps_ctx* c, const cps_step_in* in, cps_step_out* out) {
  if (!c || !in) return fail(c, CPS_ERR_ARG, "ctx and in are required");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  set_step_inputs(c, in->inletVelocity);
  int nd = 0;
  cps_step_out tmp;
  return run(c, 1, 0, 0.0, out ? out : &tmp, &nd);
}

cps_status cps_solve(cps_ctx* c, double inletVelocity, int max_outer, double eps, cps_step_out* history,
                     int* n_done) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (max_outer < 0) return fail(c, CPS_ERR_ARG, "max_outer < 0");
  if (n_done) *n_done = 0;
  if (max_outer == 0) return CPS_OK;
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  set_step_inputs(c, inletVelocity);
  return run(c, max_outer, eps > 0.0 ? 1 : 0, eps, history, n_done, nullptr, nullptr, true);
}

cps_status cps_set_inlet_ramp(cps_ctx* c, int ramp_steps) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (ramp_steps < 0) return fail(c, CPS_ERR_ARG, "ramp_steps < 0");
  c->ramp_steps = ramp_steps;
  return CPS_OK;
}

cps_status cps_set_dp_monitor(cps_ctx* c, const cps_dp_monitor* m) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  c->iter = 0;
  if (!m) {
    c->view.dpMonitor = 0;
    c->view.dpGate = 0;
    return CPS_OK;
  }
  if (m->window < 1 || m->slope_window < 0 || m->ramp_steps < 0 || !(m->percent >= 0.0))
    return fail(c, CPS_ERR_ARG, "dp monitor: window >= 1, slope_window >= 0, ramp_steps >= 0, percent >= 0");
  const size_t slots = (size_t)m->window + (size_t)(m->slope_gate ? m->slope_window : 0);
  if (slots * sizeof(double) > tile_smem_for(c->precision))
    return fail(c, CPS_ERR_ARG, "dp monitor: window + slope_window exceeds " +
                                    std::to_string(tile_smem_for(c->precision) / sizeof(double)) + " values");
  if (c->ddphist) cudaFree(c->ddphist);
  c->ddphist = nullptr;
  if (!cuda_ok(c, cudaMalloc(&c->ddphist, std::max<size_t>(slots, 1) * sizeof(double)), "cudaMalloc")) return CPS_ERR_OOM;
  if (!cuda_ok(c, cudaMemset(c->ddphist, 0, std::max<size_t>(slots, 1) * sizeof(double)), "memset")) return CPS_ERR_CUDA;
  cps::DesignView& v = c->view;
  v.dpMonitor = 1;
  v.dpGate = m->gate ? 1 : 0;
  v.dpWindow = m->window;
  v.dpSlopeGate = m->slope_gate ? 1 : 0;
  v.dpSlopeWindow = m->slope_gate ? m->slope_window : 0;
  v.dpRampSteps = m->ramp_steps;
  v.dpPercent = m->percent;
  v.dpSlopeMaxDelta = m->slope_max_delta;
  v.xPlane[0] = m->x_core_in;
  v.xPlane[1] = m->x_core_out;
  v.xPlane[2] = 0.0;
  v.xPlane[3] = (double)c->N * v.hx;  // domainXMax = N * hx (SIMPLE.cpp:250)
  v.dpHist = c->ddphist;
  return CPS_OK;
}

cps_status cps_solve_monitored(cps_ctx* c, double inletVelocity, int max_outer, double eps, cps_step_out* history,
                               double* dp_history, int* n_done, int* dp_converged) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (max_outer < 0) return fail(c, CPS_ERR_ARG, "max_outer < 0");
  if (!c->view.dpMonitor) return fail(c, CPS_ERR_ARG, "no pressure-drop monitor set (cps_set_dp_monitor)");
  if (n_done) *n_done = 0;
  if (dp_converged) *dp_converged = 0;
  if (max_outer == 0) return CPS_OK;
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  set_step_inputs(c, inletVelocity);
  return run(c, max_outer, eps > 0.0 ? 1 : 0, eps, history, n_done, dp_history, dp_converged, true);
}

cps_status cps_batch_solve(cps_ctx* const* ctxs, int n, const double* inletVelocity, const cps_batch_opts* opts,
                           cps_batch_result* results, double* kernel_ms) {
  if (!ctxs || n <= 0 || !opts || !results) return fail(nullptr, CPS_ERR_ARG, "ctxs, n > 0, opts and results required");
  if (opts->max_outer < 0) return fail(nullptr, CPS_ERR_ARG, "max_outer < 0");
  const int cl = opts->cluster_ctas > 0 ? opts->cluster_ctas : 8;
  if (cl > 16) return fail(nullptr, CPS_ERR_ARG, "cluster_ctas must be <= 16");
  cps_ctx* c0 = ctxs[0];
  for (int k = 0; k < n; ++k) {
    if (!ctxs[k]) return fail(nullptr, CPS_ERR_ARG, "NULL context in batch");
    if (ctxs[k]->device != c0->device || ctxs[k]->precision != c0->precision)
      return fail(nullptr, CPS_ERR_ARG, "a batch needs one device and one precision");
  }
  std::lock_guard<std::mutex> lock(g_batch_mutex);
  if (!cuda_ok(c0, cudaSetDevice(c0->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  std::string err;
  BatchWorkspace* ws = batch_workspace(c0->device, (size_t)n, err);
  if (!ws) return fail(c0, CPS_ERR_OOM, err);
  // The batch kernels carry the pseudo-transient term and the CFL controllers
  // only when a design of the batch has them on (a separate instantiation:
  // compiled in, they slow every batched outer iteration by a quarter).
  bool pseudo = false;
  for (int k = 0; k < n; ++k) {
    cps_ctx* c = ctxs[k];
    set_step_inputs(c, inletVelocity ? inletVelocity[k] : c->view.Uin);
    cps::BatchItem& it = ws->h_items[k];
    std::memset(&it, 0, sizeof(it));
    it.view = c->view;
    it.view.dpMonitor = 0;  // the pressure-drop monitor runs in cps_solve/cps_solve_monitored only
    it.n_outer = opts->max_outer;
    it.stop_on_conv = opts->eps > 0.0 ? 1 : 0;
    it.eps = opts->eps;
    it.hist = c->dhist;
    it.hist_cap = kHistChunk;
    it.iter0 = c->iter;
    pseudo = pseudo || c->view.pseudo != 0;
  }
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  if (opts->order_by_size)
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
      return (long long)ctxs[a]->M * ctxs[a]->N > (long long)ctxs[b]->M * ctxs[b]->N;
    });
  std::copy(ord.begin(), ord.end(), ws->h_order);
  cudaStream_t st = c0->stream;
  if (!cuda_ok(c0, cudaMemcpyAsync(ws->items, ws->h_items, sizeof(cps::BatchItem) * n, cudaMemcpyHostToDevice, st),
               "h2d") ||
      !cuda_ok(c0, cudaMemcpyAsync(ws->order, ws->h_order, sizeof(int) * n, cudaMemcpyHostToDevice, st), "h2d") ||
      !cuda_ok(c0, cudaMemsetAsync(ws->queue, 0, sizeof(int), st), "memset") ||
      !cuda_ok(c0, cudaMemsetAsync(ws->results, 0, sizeof(cps::BatchResult) * n, st), "memset"))
    return CPS_ERR_CUDA;
  if (opts->tiles_per_cta > 0) {
    // Groups sized to their designs, packed into waves (first fit, largest
    // first); one cooperative launch per wave, all CTAs of a wave co-resident.
    const void* wk = c0->precision == CPS_MIXED
                         ? (pseudo ? (const void*)cps_wave_kernel<float, true> : (const void*)cps_wave_kernel<float, false>)
                         : (pseudo ? (const void*)cps_wave_kernel<double, true> : (const void*)cps_wave_kernel<double, false>);
    int per_sm = 0, sms = 0;
    const size_t tsm = tile_smem_for(c0->precision);
    if (!allow_smem(c0, wk, tsm) ||
        !cuda_ok(c0, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wk, cps::kThreads, tsm), "occupancy") ||
        !cuda_ok(c0, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c0->device), "attribute"))
      return CPS_ERR_CUDA;
    const int max_ctas = std::min(sms * per_sm, kMaxGridCtas);
    if (max_ctas < 1) return fail(c0, CPS_ERR_CUDA, "wave kernel does not fit on an SM");
    std::vector<int> ctas(n);
    for (int k = 0; k < n; ++k) {
      const long long tiles = (long long)((ctxs[k]->M - 1 + cps::kTileI - 1) / cps::kTileI) *
                              ((ctxs[k]->N - 1 + cps::kTileJ - 1) / cps::kTileJ);
      ctas[k] = (int)std::max(1LL, std::min<long long>(max_ctas, (tiles + opts->tiles_per_cta - 1) / opts->tiles_per_cta));
    }
    std::vector<int> byc(n);
    std::iota(byc.begin(), byc.end(), 0);
    std::stable_sort(byc.begin(), byc.end(), [&](int a, int b) { return ctas[a] > ctas[b]; });
    std::vector<std::vector<int>> waves;
    std::vector<int> room;
    for (int k : byc) {
      size_t w = 0;
      while (w < waves.size() && room[w] < ctas[k]) ++w;
      if (w == waves.size()) { waves.emplace_back(); room.push_back(max_ctas); }
      waves[w].push_back(k);
      room[w] -= ctas[k];
    }
    // plan: for each wave, first[G + 1] then which[G]; at most 3n ints
    std::vector<size_t> at(waves.size());
    size_t pos = 0;
    for (size_t w = 0; w < waves.size(); ++w) {
      at[w] = pos;
      int* f = ws->h_plan + pos;
      const int G = (int)waves[w].size();
      f[0] = 0;
      for (int q = 0; q < G; ++q) {
        f[q + 1] = f[q] + ctas[waves[w][q]];
        f[G + 1 + q] = waves[w][q];
      }
      pos += 2 * (size_t)G + 1;
    }
    if (!cuda_ok(c0, cudaMemcpyAsync(ws->plan, ws->h_plan, sizeof(int) * pos, cudaMemcpyHostToDevice, st), "h2d"))
      return CPS_ERR_CUDA;
    const cps::BatchItem* items = ws->items;
    cps::BatchResult* res = ws->results;
    if (!cuda_ok(c0, cudaEventRecord(ws->ev0, st), "event")) return CPS_ERR_CUDA;
    for (size_t w = 0; w < waves.size(); ++w) {
      int G = (int)waves[w].size();
      const int* first = ws->plan + at[w];
      const int* which = first + G + 1;
      const int grid = ws->h_plan[at[w] + G];
      if (!cuda_ok(c0, cudaMemsetAsync(ws->bars, 0, sizeof(cps::GridBarrier) * G, st), "memset")) return CPS_ERR_CUDA;
      void* args[] = {&items, &first, &which, &G, &res, &ws->bars, &ws->rings};
      if (!cuda_ok(c0, cudaLaunchCooperativeKernel(wk, dim3(grid), dim3(cps::kThreads), args, tsm, st),
                   "cooperative wave launch"))
        return CPS_ERR_CUDA;
    }
  } else if (opts->group_ctas > 0) {
    // Groups of CTAs in one cooperative launch (all CTAs co-resident).
    const void* gk = c0->precision == CPS_MIXED
                         ? (pseudo ? (const void*)cps_group_kernel<float, true> : (const void*)cps_group_kernel<float, false>)
                         : (pseudo ? (const void*)cps_group_kernel<double, true> : (const void*)cps_group_kernel<double, false>);
    int per_sm = 0, sms = 0;
    const size_t tsm = tile_smem_for(c0->precision);
    if (!allow_smem(c0, gk, tsm) ||
        !cuda_ok(c0, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gk, cps::kThreads, tsm), "occupancy") ||
        !cuda_ok(c0, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c0->device), "attribute"))
      return CPS_ERR_CUDA;
    const int K = opts->group_ctas;
    const int max_ctas = std::min(sms * per_sm, kMaxGridCtas);
    if (K > max_ctas) return fail(c0, CPS_ERR_ARG, "group_ctas exceeds the co-resident CTAs of the device");
    int groups = std::min(max_ctas / K, n);
    if (opts->max_clusters > 0) groups = std::min(groups, opts->max_clusters);
    groups = std::max(groups, 1);
    if (!cuda_ok(c0, cudaMemsetAsync(ws->bars, 0, sizeof(cps::GridBarrier) * groups, st), "memset") ||
        !cuda_ok(c0, cudaMemsetAsync(ws->slots, 0, sizeof(int) * 2 * groups, st), "memset"))
      return CPS_ERR_CUDA;
    const cps::BatchItem* items = ws->items;
    const int* order = ws->order;
    int* queue = ws->queue;
    cps::BatchResult* res = ws->results;
    int nn = n, kk = K;
    void* args[] = {&items, &order, &nn, &queue, &res, &ws->bars, &ws->rings, &ws->slots, &kk};
    if (!cuda_ok(c0, cudaEventRecord(ws->ev0, st), "event")) return CPS_ERR_CUDA;
    if (!cuda_ok(c0, cudaLaunchCooperativeKernel(gk, dim3(groups * K), dim3(cps::kThreads), args, tsm, st),
                 "cooperative group launch"))
      return CPS_ERR_CUDA;
  } else {
  using KernFn = void (*)(const cps::BatchItem*, const int*, int, int*, cps::BatchResult*);
  KernFn kern = c0->precision == CPS_MIXED
                    ? (pseudo ? (KernFn)cps_cluster_kernel<float, true> : (KernFn)cps_cluster_kernel<float, false>)
                    : (pseudo ? (KernFn)cps_cluster_kernel<double, true> : (KernFn)cps_cluster_kernel<double, false>);
  if (cl > 8 &&
      !cuda_ok(c0, cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1), "attr"))
    return CPS_ERR_CUDA;
  if (!allow_smem(c0, (const void*)kern, tile_smem_for(c0->precision))) return CPS_ERR_CUDA;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(cps::kThreads);
  cfg.dynamicSmemBytes = tile_smem_for(c0->precision);
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(cl * 64);
  int max_clusters = 0;
  if (!cuda_ok(c0, cudaOccupancyMaxActiveClusters(&max_clusters, (const void*)kern, &cfg), "cluster occupancy"))
    return CPS_ERR_CUDA;
  if (max_clusters < 1) return fail(c0, CPS_ERR_CUDA, "cluster configuration does not fit");
  int clusters = std::min(max_clusters, n);
  if (opts->max_clusters > 0) clusters = std::min(clusters, opts->max_clusters);
  cfg.gridDim = dim3(cl * clusters);
  const cps::BatchItem* items = ws->items;
  const int* order = ws->order;
  int* queue = ws->queue;
  cps::BatchResult* res = ws->results;
  if (!cuda_ok(c0, cudaEventRecord(ws->ev0, st), "event")) return CPS_ERR_CUDA;
  if (!cuda_ok(c0, cudaLaunchKernelEx(&cfg, kern, items, order, n, queue, res), "cluster launch")) return CPS_ERR_CUDA;
  }
  if (!cuda_ok(c0, cudaEventRecord(ws->ev1, st), "event") ||
      !cuda_ok(c0, cudaMemcpyAsync(ws->h_results, ws->results, sizeof(cps::BatchResult) * n, cudaMemcpyDeviceToHost,
                                   st), "d2h") ||
      !cuda_ok(c0, cudaStreamSynchronize(st), "batch kernel"))
    return CPS_ERR_CUDA;
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ws->ev0, ws->ev1);
  if (kernel_ms) *kernel_ms = ms;
  cps_status status = CPS_OK;
  for (int k = 0; k < n; ++k) {
    const cps::BatchResult& r = ws->h_results[k];
    results[k].n_done = r.n_done;
    results[k].converged = r.converged;
    results[k].status = r.status == cps::kStatusOk        ? CPS_OK
                        : r.status == cps::kStatusTimeout ? CPS_ERR_TIMEOUT
                                                          : CPS_ERR_DIVERGED;
    to_step_out(r.last, &results[k].last);
    ctxs[k]->outer_done += r.n_done;
    ctxs[k]->iter += r.n_done;
    if (r.status != cps::kStatusOk) {
      status = (cps_status)results[k].status;
      ctxs[k]->err = r.status == cps::kStatusTimeout ? "device group barrier timed out"
                                                     : "residual is not finite (solution diverged)";
    }
  }
  c0->kernel_ms += ms;
  c0->launches += 1;
  if (status != CPS_OK) g_create_error = "at least one design diverged; see results[k].status";
  return status;
}

cps_status cps_get_history(cps_ctx* c, int n, cps_step_out* history) {
  if (!c || !history || n < 0 || n > kHistChunk) return fail(c, CPS_ERR_ARG, "bad history request");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  if (n == 0) return CPS_OK;
  if (!cuda_ok(c, cudaMemcpyAsync(c->hhist, c->dhist, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost, c->stream),
               "d2h") ||
      !cuda_ok(c, cudaStreamSynchronize(c->stream), "sync"))
    return CPS_ERR_CUDA;
  for (int k = 0; k < n; ++k) to_step_out(c->hhist + (size_t)8 * k, &history[k]);
  return CPS_OK;
}

cps_status cps_sample_plane(cps_ctx* c, double x, cps_plane* out) {
  if (!c || !out) return fail(c, CPS_ERR_ARG, "ctx and out are required");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  cps_plane_kernel<<<1, cps::kThreads, 0, c->stream>>>(c->view, x, c->dplane);
  if (!cuda_ok(c, cudaGetLastError(), "plane launch")) return CPS_ERR_CUDA;
  if (!cuda_ok(c, cudaMemcpyAsync(c->hhist, c->dplane, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h") ||
      !cuda_ok(c, cudaStreamSynchronize(c->stream), "plane"))
    return CPS_ERR_CUDA;
  out->flowArea = c->hhist[0]; out->massFlux = c->hhist[1]; out->avgStatic = c->hhist[2];
  out->avgDynamic = c->hhist[3]; out->avgTotal = c->hhist[4]; out->valid = c->hhist[5] != 0.0;
  return CPS_OK;
}

cps_status cps_download_fields(cps_ctx* c, double* u, double* v, double* p, double* pStar, double* uStar,
                               double* vStar, double* dE, double* dN, int layout) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (layout != CPS_ROW_MAJOR && layout != CPS_COL_MAJOR) return fail(c, CPS_ERR_ARG, "bad layout");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  const int M = c->M, N = c->N;
  const cps::DesignView& w = c->view;
  if (!download_plane(c, u, w.u, M + 1, N, layout) || !download_plane(c, v, w.v, M, N + 1, layout) ||
      !download_plane(c, p, w.p, M + 1, N + 1, layout) || !download_plane(c, pStar, w.pc, M + 1, N + 1, layout) ||
      !download_plane(c, uStar, w.us, M + 1, N, layout) || !download_plane(c, vStar, w.vs, M, N + 1, layout) ||
      !download_plane(c, dE, w.dE, M + 1, N, layout) || !download_plane(c, dN, w.dN, M, N + 1, layout))
    return CPS_ERR_CUDA;
  return CPS_OK;
}

}  // extern "C"
