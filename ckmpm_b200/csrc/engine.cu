// Host side of the B200 CK-MPM engine: scene/model lifetime, device memory,
// setup, CUDA-graph substep replay and the C ABI declared in include/ckmpm.h.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/ckmpm.h"
#include "kernels.cuh"

using namespace ckmpm;

namespace {

constexpr int kFusedThreads = 256;
constexpr int kProbeThreads = 256;
constexpr int kGraphChunk = 8;
// Default substeps between re-layouts of each block's particles into the setup
// order (reorder_gather_kernel): a re-layout moves the whole state twice, and
// the layout keeps most of its effect for a few hundred substeps (sand column:
// the fused launch 3-7 % shorter than with particles in input order through
// 3200 substeps at 128, against none after 1600 with the setup order alone).
constexpr uint32_t kReorderEvery = 128;
constexpr int kMaxGraphChunk = 64;
constexpr int kMixedKind = 7;  // ModelHost::mat.kind of a batch's single model (per-scene materials)
constexpr const char* kVersion = "ckmpm-b200 0.2.0";

thread_local std::string g_create_error;

struct ModelHost {
  ckmpm_material mat{};
  float mass = 0.f, vol = 0.f;
  uint32_t n = 0;       // particles passed in
  uint32_t n_valid = 0; // particles binned at setup
  uint32_t nv = 0;
  ModelDev dev{};
  uint32_t ntiles = 0;
  // The model's I/O arena: one device allocation made by ckmpm_add_model /
  // ckmpm_add_batch and kept until ckmpm_destroy.  Until setup it holds the
  // inputs (x in ox, v in ov) and, during setup, the binning sort's keys and
  // values (in oF) and its scratch; afterwards the export buffers.
  unsigned char* io = nullptr;
  float* ox = nullptr;
  float* ov = nullptr;
  float* oF = nullptr;
  float* oaux = nullptr;
  uint32_t* oid = nullptr;
  uint32_t* oflag = nullptr;  // input-order export: live flags by id, then their exclusive scan
  uint32_t* opos = nullptr;
  uint32_t* oscan = nullptr;  // the export scan's tile sums (scan_tiles(n) words)
  // Asynchronous export: recorded on the copy stream after this model's
  // staging buffer has been copied out.
  cudaEvent_t ev_copied = nullptr;
  bool copy_pending = false;
  // Batch: per-scene materials and input offsets (host copies and device arrays).
  std::vector<SceneMat> smat;
  std::vector<uint32_t> sstart;
  std::vector<int32_t> skind;
};

}  // namespace

struct ckmpm_scene {
  ckmpm_scene_desc desc{};
  SceneDev sc{};
  std::vector<ModelHost> models;
  GridDev grid{};
  Scalars* scal = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  bool setup_done = false;
  std::string err;
  int sm_count = 0;
  int fused_ctas = 0;
  int occ[4] = {0, 0, 0, 0};  // resident fused CTAs per SM at 128 / 256 / 1024 / 192 threads
  uint32_t nstack = 1;     // stacked domains: 1, or the scene count of a batch
  ckmpm_tuning tune{};
  // Every device allocation with its size; the first n_state_allocs hold the
  // simulation state (what a checkpoint copies), later ones are export buffers.
  std::vector<std::pair<void*, size_t>> allocs;
  size_t n_state_allocs = 0;
  cudaGraphExec_t graph_chunk = nullptr;
  cudaGraphExec_t graph_one = nullptr;
  uint64_t host_step = 0;
  // Substeps between re-layouts of the particles (reorder_gather_kernel); 0 = never.
  uint32_t reorder_every = kReorderEvery;
  uint64_t last_reorder = 0;
  // Asynchronous position export: copy stream, its events, the live count
  // (pinned host scalar) and whether a copy may still be in flight.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_probe = nullptr, ev_copy = nullptr;
  uint32_t* export_count = nullptr;
  bool export_pending = false;
  uint32_t rigid_count = 0;       // leading rigid particles of every von Mises model
  float rigid_v[3] = {0.f, 0.f, 0.f};
};

namespace {

ckmpm_status fail(ckmpm_scene* s, ckmpm_status code, const std::string& msg) {
  if (s) s->err = msg;
  else g_create_error = msg;
  return code;
}

#define CK_CUDA(s, call)                                                                              \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      return fail((s), CKMPM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));           \
  } while (0)

// Consecutive sub-allocations of one device allocation, each on a 256-byte
// boundary.  With a null base it only measures: run a layout once to size the
// allocation, then again on the allocation to place the pointers.
struct Carve {
  unsigned char* base = nullptr;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    off = (off + 255) & ~static_cast<size_t>(255);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += std::max<size_t>(count, 1) * sizeof(T);
    return p;
  }
};

template <typename T>
cudaError_t dalloc(ckmpm_scene* s, T** p, size_t count) {
  void* q = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e == cudaSuccess) s->allocs.emplace_back(q, bytes);
  *p = static_cast<T*>(q);
  return e;
}

void free_graphs(ckmpm_scene* s) {
  if (s->graph_chunk) cudaGraphExecDestroy(s->graph_chunk);
  if (s->graph_one) cudaGraphExecDestroy(s->graph_one);
  s->graph_chunk = s->graph_one = nullptr;
}

template <int KIND, int NT, bool RIGID>
cudaError_t launch_fused(ckmpm_scene* s, const ModelHost& m) {
  g2p2g_kernel<KIND, NT, RIGID><<<s->fused_ctas, NT, kSmemFused, s->stream>>>(s->sc, m.dev, s->grid, s->scal);
  return cudaGetLastError();
}

template <int NT, bool RIGID>
cudaError_t launch_fused_kind(ckmpm_scene* s, const ModelHost& m) {
  switch (m.mat.kind) {
    case CKMPM_FIXED_COROTATED: return launch_fused<kFixedCorotated, NT, RIGID>(s, m);
    case CKMPM_LINEAR: return launch_fused<kLinear, NT, RIGID>(s, m);
    case CKMPM_DRUCKER_PRAGER: return launch_fused<kDruckerPrager, NT, RIGID>(s, m);
    case CKMPM_VON_MISES: return launch_fused<kVonMises, NT, RIGID>(s, m);
    case CKMPM_NACC: return launch_fused<kNacc, NT, RIGID>(s, m);
    default: return launch_fused<kFluid, NT, RIGID>(s, m);
  }
}

template <int NT>
cudaError_t launch_fused_nt(ckmpm_scene* s, const ModelHost& m) {
  if (m.mat.kind == kMixedKind) return launch_fused<kMixed, NT, false>(s, m);  // batches have no rigid particles
  return s->sc.rigid ? launch_fused_kind<NT, true>(s, m) : launch_fused_kind<NT, false>(s, m);
}

cudaError_t launch_fused_any(ckmpm_scene* s, const ModelHost& m) {
  switch (s->tune.threads) {
    case 128: return launch_fused_nt<128>(s, m);
    case 192: return launch_fused_nt<192>(s, m);
    case 1024: return launch_fused_nt<1024>(s, m);
    default: return launch_fused_nt<256>(s, m);
  }
}

// Index of a CTA size in ckmpm_scene::occ (-1 for a size that has no kernel).
int shape_index(uint32_t threads) {
  return threads == 128 ? 0 : threads == 256 ? 1 : threads == 1024 ? 2 : threads == 192 ? 3 : -1;
}

template <int NT>
cudaError_t set_fused_attributes(int* occ) {
  const void* fns[13] = {reinterpret_cast<const void*>(g2p2g_kernel<kFixedCorotated, NT>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kLinear, NT>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kDruckerPrager, NT>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kFluid, NT>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kVonMises, NT>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kNacc, NT>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kMixed, NT>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kFixedCorotated, NT, true>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kLinear, NT, true>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kDruckerPrager, NT, true>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kFluid, NT, true>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kVonMises, NT, true>),
                         reinterpret_cast<const void*>(g2p2g_kernel<kNacc, NT, true>)};
  int lowest = 1 << 30;
  for (const void* fn : fns) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSmemFused));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, NT, kSmemFused);
    if (e != cudaSuccess) return e;
    lowest = std::min(lowest, o);
  }
  *occ = std::max(1, lowest);
  return cudaSuccess;
}

// The fused and rasterisation kernels' attributes belong to the process and the
// device, not to a scene: they are set, and the fused kernels' occupancy at
// 128 / 256 / 1024 / 192 threads queried (52 kernel variants), once per device,
// by the first scene created on it.  A failure is not cached.
std::mutex g_attr_mutex;
std::map<int, std::array<int, 4>> g_attr_occ;

cudaError_t fused_attributes(int device, int* occ4) {
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  auto it = g_attr_occ.find(device);
  if (it == g_attr_occ.end()) {
    std::array<int, 4> occ{0, 0, 0, 0};
    cudaError_t e = set_fused_attributes<128>(&occ[0]);
    if (e == cudaSuccess) e = set_fused_attributes<256>(&occ[1]);
    if (e == cudaSuccess) e = set_fused_attributes<1024>(&occ[2]);
    if (e == cudaSuccess) e = set_fused_attributes<192>(&occ[3]);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(reinterpret_cast<const void*>(rasterize_kernel<kFusedThreads>),
                               cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSmemFused));
    if (e != cudaSuccess) return e;
    it = g_attr_occ.emplace(device, occ).first;
  }
  for (int k = 0; k < 4; ++k) occ4[k] = it->second[k];
  return cudaSuccess;
}

// Compaction of one model's next block list into list `out`.
cudaError_t launch_compact(ckmpm_scene* s, const ModelHost& m, const BlockListDev& out) {
  compact_reduce_kernel<<<m.ntiles, kCompactThreads, 0, s->stream>>>(s->sc, m.dev.dense_total, m.dev.tile_sums);
  compact_scatter_kernel<<<m.ntiles, kCompactThreads, 0, s->stream>>>(s->sc, m.dev.dense_total, m.dev.tile_sums, out,
                                                                       m.dev.cap_slots, m.dev.ticket, s->scal);
  return cudaGetLastError();
}

__global__ void set_next_dt_kernel(Scalars* scal, float dt) {
  if (threadIdx.x == 0) {
    scal->next_dt = dt;
    scal->next_dt_d = static_cast<double>(dt);
  }
}

__global__ void set_frame_end_kernel(Scalars* scal, double frame_time) {
  if (threadIdx.x == 0) scal->frame_end = scal->time + frame_time;
}

// Zero (and stamp with step + epoch_offset) the blocks of grid[grid_parity]
// that a substep over block lists bl[list_parity] deposits into.
cudaError_t launch_zero(ckmpm_scene* s, int list_parity, int grid_parity, int32_t epoch_offset) {
  for (auto& m : s->models)
    zero_windows_kernel<<<s->sm_count * 4, 256, 0, s->stream>>>(s->sc, m.dev.bl[list_parity],
                                                                 s->grid.grid[grid_parity],
                                                                 s->grid.stamp[grid_parity], s->scal, epoch_offset);
  return cudaGetLastError();
}

// Enqueue one substep for every model.  The compaction of each model writes
// the block list the fused kernel did not read: that of the other parity.
// Once every model's fused kernel has read grid[parity], its blocks that the
// next substep deposits into are zeroed for it (epoch step + 2).
cudaError_t enqueue_substep(ckmpm_scene* s, int parity_of_step) {
  for (auto& m : s->models) {
    cudaError_t e = launch_fused_any(s, m);
    if (e != cudaSuccess) return e;
    e = launch_compact(s, m, m.dev.bl[parity_of_step ^ 1]);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = launch_zero(s, parity_of_step ^ 1, parity_of_step, 2);
  if (e != cudaSuccess) return e;
  end_substep_kernel<<<1, 32, 0, s->stream>>>(s->scal);
  return cudaGetLastError();
}

cudaError_t build_graph(ckmpm_scene* s, int nsub, int first_parity, cudaGraphExec_t* exec) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  for (int i = 0; i < nsub; ++i) {
    e = enqueue_substep(s, (first_parity + i) & 1);
    if (e != cudaSuccess) break;
  }
  cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return e;
  }
  if (e2 != cudaSuccess) return e2;
  e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  return e;
}

// Material kinds this engine runs and the parameter each needs to be positive.
bool valid_material(const ckmpm_material& m, std::string* why) {
  switch (m.kind) {
    case CKMPM_FIXED_COROTATED:
    case CKMPM_LINEAR:
    case CKMPM_DRUCKER_PRAGER:
      if (!(m.p[1] > 0.f)) return (*why = "mu (p[1]) must be positive", false);
      return true;
    case CKMPM_VON_MISES:
    case CKMPM_NACC:
      if (!(m.p[0] > 0.f)) return (*why = "mu (p[0]) must be positive", false);
      return true;
    case CKMPM_FLUID:
      return true;
    default:
      return (*why = "unsupported material kind", false);
  }
}

// Initial aux value: J0 for the fluid, alpha0 (the initial logJp) for NACC, else 0.
float initial_aux(const ckmpm_material& m) {
  if (m.kind == CKMPM_VON_MISES) return 1.f;  // the rigid flag: deformable
  return m.kind == CKMPM_FLUID ? m.p[3] : (m.kind == CKMPM_NACC ? m.p[2] : 0.f);
}

ckmpm_status status_from(ckmpm_scene* s, const Scalars& h) {
  if (h.status & kStatusTimeout) return fail(s, CKMPM_ERR_TIMEOUT, "a bounded device wait gave up");
  if (h.status & kStatusCapacity)
    return fail(s, CKMPM_ERR_CAPACITY, "block capacity exceeded (particles per block or block table)");
  if (h.status & kStatusNumeric) return fail(s, CKMPM_ERR_NUMERIC, "non-finite or out-of-range P2G contribution");
  if (h.status & kStatusConsistency) return fail(s, CKMPM_ERR_INVALID, "rebin consistency check failed");
  if (h.status & kStatusOutsideBlock)
    return fail(s, CKMPM_ERR_NUMERIC, "a particle was outside the stencil window of its block");
  return CKMPM_OK;
}

// Page-locked host words (each scene's export live count), handed out from
// slabs of 1024 shared by the process: page-locking is a system call that took
// 1.5 to 6 ms per cudaMallocHost, as long as the rest of a scene's creation.
// The slabs are portable (usable from every device's context) and live as long
// as the process; a destroyed scene returns its word.
std::mutex g_pin_mutex;
std::vector<uint32_t*> g_pin_free;

uint32_t* pinned_word() {
  constexpr size_t kWords = 1024, kStride = 16;  // one word per 64 bytes
  std::lock_guard<std::mutex> lock(g_pin_mutex);
  if (g_pin_free.empty()) {
    void* slab = nullptr;
    if (cudaHostAlloc(&slab, kWords * kStride * sizeof(uint32_t), cudaHostAllocPortable) != cudaSuccess)
      return nullptr;
    for (size_t i = kWords; i-- > 0;) g_pin_free.push_back(static_cast<uint32_t*>(slab) + i * kStride);
  }
  uint32_t* w = g_pin_free.back();
  g_pin_free.pop_back();
  return w;
}

void release_pinned_word(uint32_t* w) {
  std::lock_guard<std::mutex> lock(g_pin_mutex);
  g_pin_free.push_back(w);
}

ckmpm_status create_impl(const ckmpm_scene_desc* desc, uint32_t nstack, ckmpm_scene** out) {
  if (!desc || !out) return fail(nullptr, CKMPM_ERR_INVALID, "null argument");
  *out = nullptr;
  if (nstack < 1 || nstack > CKMPM_MAX_BATCH_SCENES) return fail(nullptr, CKMPM_ERR_INVALID, "scene count out of range");
  if (!(desc->dx > 0.f)) return fail(nullptr, CKMPM_ERR_INVALID, "dx must be positive");
  for (int a = 0; a < 3; ++a)
    if (desc->domain_blocks[a] < 1 || desc->domain_blocks[a] > 4096)
      return fail(nullptr, CKMPM_ERR_INVALID, "domain_blocks out of range");
  const uint64_t nbd = static_cast<uint64_t>(desc->domain_blocks[0]) * desc->domain_blocks[1] * desc->domain_blocks[2];
  if (nbd * nstack > (1ull << 28)) return fail(nullptr, CKMPM_ERR_INVALID, "domain too large for the dense block table");
  if (desc->boundary != CKMPM_BOUNDARY_STICKY_BLOCKS && desc->boundary != CKMPM_BOUNDARY_SLIP_FLOOR &&
      desc->boundary != CKMPM_BOUNDARY_FIELD)
    return fail(nullptr, CKMPM_ERR_INVALID, "unknown boundary kind");
  if (desc->max_particles_per_block > static_cast<uint32_t>(kMaxParticlesPerBlock))
    return fail(nullptr, CKMPM_ERR_INVALID, "max_particles_per_block > 4096");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, CKMPM_ERR_CUDA, "no CUDA device is available");
  if (desc->device < 0 || desc->device >= ndev) return fail(nullptr, CKMPM_ERR_INVALID, "bad device ordinal");

  ckmpm_scene* s = new ckmpm_scene();
  s->desc = *desc;
  s->nstack = nstack;
  if (s->desc.max_particles_per_block == 0) s->desc.max_particles_per_block = kMaxParticlesPerBlock;
  auto bail = [&](ckmpm_status st) {
    g_create_error = s->err;
    ckmpm_destroy(s);
    return st;
  };
  if (cudaSetDevice(desc->device) != cudaSuccess) return bail(fail(s, CKMPM_ERR_CUDA, "cudaSetDevice failed"));
  cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, desc->device);
  if (cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(s, CKMPM_ERR_CUDA, "cudaStreamCreate failed"));
  s->stream = s->own_stream;
  // Asynchronous position export: its copy stream, events and pinned live count.
  if (cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_probe, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_copy, cudaEventDisableTiming) != cudaSuccess ||
      (s->export_count = pinned_word()) == nullptr)
    return bail(fail(s, CKMPM_ERR_CUDA, "export stream, events or pinned count could not be created"));
  *s->export_count = 0;

  SceneDev& sc = s->sc;
  sc.dx = desc->dx;
  sc.inv_dx = static_cast<float>(1.0 / static_cast<double>(desc->dx));
  for (int a = 0; a < 3; ++a) sc.dims[a] = desc->domain_blocks[a];
  sc.gravity = desc->gravity;
  sc.mass_clamp = desc->mass_clamp;
  sc.boundary = desc->boundary;
  sc.floor_cells = desc->floor_cells;
  init_colour_classes(sc, nstack);
  const uint64_t nbt = sc.nblocks_domain;

  // Dense grids, stamps, the scalars and (with a boundary field) the per-cell
  // rules, in one device allocation: each cudaMalloc maps pages of its own,
  // and on a 64^3-block domain one call for all of them took 0.4 ms where five
  // took 2 ms.  The rules start FREE until ckmpm_set_boundary_field; a batch's
  // scenes share the one field of their common domain extent.
  const bool field = desc->boundary == CKMPM_BOUNDARY_FIELD;
  const size_t cells = static_cast<size_t>(nbd) * 64;
  uint8_t* rule = nullptr;
  float* param = nullptr;
  auto scene_layout = [&](Carve& c) {
    for (int b = 0; b < 2; ++b) s->grid.grid[b] = c.take<long long>(static_cast<size_t>(nbt) * 512);
    for (int b = 0; b < 2; ++b) s->grid.stamp[b] = c.take<int32_t>(nbt);
    s->scal = c.take<Scalars>(1);
    if (field) {
      rule = c.take<uint8_t>(cells);
      param = c.take<float>(3 * cells);
    }
  };
  Carve scene_size;
  scene_layout(scene_size);
  Carve scene_place;
  if (dalloc(s, &scene_place.base, scene_size.off) != cudaSuccess)
    return bail(fail(s, CKMPM_ERR_CUDA, "grid allocation failed"));
  scene_layout(scene_place);
  for (int b = 0; b < 2; ++b) cudaMemsetAsync(s->grid.stamp[b], 0xFF, sizeof(int32_t) * nbt, s->stream);
  cudaMemsetAsync(s->scal, 0, sizeof(Scalars), s->stream);
  if (field) {
    cudaMemsetAsync(rule, 0, cells, s->stream);
    cudaMemsetAsync(param, 0, sizeof(float) * 3 * cells, s->stream);
    sc.brule = rule;
    sc.bparam = param;
  }

  if (fused_attributes(desc->device, s->occ) != cudaSuccess)
    return bail(fail(s, CKMPM_ERR_CUDA, "cudaFuncSetAttribute failed"));
  // Default launch shape: 256 threads, as many resident CTAs as fit, graphs of 8.
  s->tune.threads = kFusedThreads;
  s->tune.ctas_per_sm = static_cast<uint32_t>(s->occ[1]);
  s->tune.graph_chunk = kGraphChunk;
  s->tune.probe_ms = 0.f;
  s->fused_ctas = s->occ[1] * s->sm_count;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return bail(fail(s, CKMPM_ERR_CUDA, "init sync failed"));
  *out = s;
  return CKMPM_OK;
}

ckmpm_status apply_tuning(ckmpm_scene* s, const ckmpm_tuning& t) {
  if (shape_index(t.threads) < 0) return fail(s, CKMPM_ERR_INVALID, "threads must be 128, 192, 256 or 1024");
  const int occ = s->occ[shape_index(t.threads)];
  if (t.ctas_per_sm < 1 || t.ctas_per_sm > static_cast<uint32_t>(occ))
    return fail(s, CKMPM_ERR_INVALID, "ctas_per_sm must be between 1 and the kernel's occupancy");
  if (t.graph_chunk < 2 || t.graph_chunk > kMaxGraphChunk || (t.graph_chunk & 1))
    return fail(s, CKMPM_ERR_INVALID, "graph_chunk must be even, 2..64");
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_graphs(s);
  s->tune = t;
  s->fused_ctas = static_cast<int>(t.ctas_per_sm) * s->sm_count;
  return CKMPM_OK;
}

// Checkpoint: the state allocations back to back, each at a 256-byte offset.
size_t checkpoint_bytes(const ckmpm_scene* s) {
  size_t total = 0;
  for (size_t i = 0; i < s->n_state_allocs; ++i) total += (s->allocs[i].second + 255) & ~static_cast<size_t>(255);
  return total;
}

cudaError_t checkpoint_copy(ckmpm_scene* s, unsigned char* buf, bool save) {
  size_t off = 0;
  for (size_t i = 0; i < s->n_state_allocs; ++i) {
    void* p = s->allocs[i].first;
    const size_t b = s->allocs[i].second;
    cudaError_t e = save ? cudaMemcpyAsync(buf + off, p, b, cudaMemcpyDeviceToDevice, s->stream)
                         : cudaMemcpyAsync(p, buf + off, b, cudaMemcpyDeviceToDevice, s->stream);
    if (e != cudaSuccess) return e;
    off += (b + 255) & ~static_cast<size_t>(255);
  }
  return cudaSuccess;
}

}  // namespace

// Places the I/O arena of a model (see ModelHost::io): export buffers for
// n particles, with the setup sort's four key/value arrays inside oF, the
// sort's and the export scan's scratch after them.
static void io_layout(ModelHost& m, bool track, Carve& c) {
  const size_t n = m.n;
  m.ox = c.take<float>(3 * n);
  m.ov = c.take<float>(3 * n);
  m.oF = c.take<float>(9 * n);
  m.oaux = c.take<float>(n);
  m.oid = c.take<uint32_t>(n);
  m.oflag = track ? c.take<uint32_t>(n) : nullptr;
  m.opos = track ? c.take<uint32_t>(n) : nullptr;
  m.oscan = track ? c.take<uint32_t>(scan_tiles(static_cast<uint32_t>(n))) : nullptr;
}

// Places a model's simulation state: the double-buffered particle arrays and
// block lists, the binning totals, compaction partials, the work ticket, the
// sorted initial velocities and a batch's per-scene tables.
static void state_layout(ModelHost& m, uint32_t nbd, bool track, Carve& c) {
  ModelDev& d = m.dev;
  const size_t n = m.n;
  const bool batch = m.mat.kind == kMixedKind;
  const bool hasF = batch || material_has_F(m.mat.kind);
  const bool hasAux = batch || material_has_aux(m.mat.kind);
  const bool hasQ = batch ? std::count(m.skind.begin(), m.skind.end(), CKMPM_LINEAR) > 0 : m.mat.kind == CKMPM_LINEAR;
  for (int b = 0; b < 2; ++b) {
    StateDev& st = d.st[b];
    for (int a = 0; a < 3; ++a) st.x[a] = c.take<float>(n);
    for (int k = 0; k < 9; ++k) st.F[k] = hasF ? c.take<float>(n) : nullptr;
    st.aux = hasAux ? c.take<float>(n) : nullptr;
    for (int k = 0; k < 9; ++k) st.Q[k] = hasQ ? c.take<float>(n) : nullptr;
    st.id = track ? c.take<uint32_t>(n) : nullptr;
    BlockListDev& bl = d.bl[b];
    bl.keys = c.take<int4>(d.cap_slots);
    bl.start = c.take<uint32_t>(d.cap_slots);
    bl.count = c.take<uint32_t>(d.cap_slots);
    bl.table = c.take<int32_t>(nbd);
    bl.prefix28 = c.take<uint32_t>(static_cast<size_t>(d.cap_slots) * 28);
    bl.idx = c.take<uint16_t>(n);
    bl.nblocks = c.take<uint32_t>(1);
    bl.nparticles = c.take<uint32_t>(1);
  }
  d.dense_total = c.take<uint32_t>(nbd);
  d.tile_sums = c.take<uint32_t>(2 * static_cast<size_t>(m.ntiles));
  d.ticket = c.take<uint32_t>(1);
  d.vel_in = c.take<float>(3 * n);
  d.smat = batch ? c.take<SceneMat>(m.smat.size()) : nullptr;
  d.sstart = batch ? c.take<uint32_t>(m.sstart.size()) : nullptr;
}

// Makes the model's state arena: all of its state in one allocation, one entry
// of s->allocs, so checkpoints copy it whole.  Its size depends only on the
// particle count, the domain and the scene's flags, all known when the model
// is added.
static cudaError_t alloc_state(ckmpm_scene* s, ModelHost& m) {
  ModelDev& d = m.dev;
  const uint32_t nbd = s->sc.nblocks_domain;
  const bool track = m.mat.kind == kMixedKind || (s->desc.flags & CKMPM_FLAG_TRACK_IDS) != 0;
  d.cap_particles = m.n;
  d.cap_slots = std::max<uint32_t>(1, std::min<uint32_t>(nbd, m.n));
  m.ntiles = (nbd + kCompactTile - 1) / kCompactTile;
  Carve size;
  state_layout(m, nbd, track, size);
  void* arena = nullptr;
  cudaError_t e = cudaMalloc(&arena, size.off);
  if (e != cudaSuccess) return e;
  s->allocs.emplace_back(arena, size.off);
  Carve place{static_cast<unsigned char*>(arena), 0};
  state_layout(m, nbd, track, place);
  return cudaSuccess;
}

// Setup's work arrays, three of n u32 inside oF (9 n floats): 0 the particles'
// flat block indices, 1 the per-slot placement cursors, 2 the particle order.
static uint32_t* sort_array(const ModelHost& m, int k) {
  return reinterpret_cast<uint32_t*>(m.oF) + static_cast<size_t>(k) * m.n;
}

// Makes the model's I/O arena and copies its input positions and velocities
// into it (DMA when the caller's buffers are pinned), then waits, so the
// caller may reuse its buffers on return and ckmpm_setup reads the inputs
// from device memory.
static cudaError_t stage_inputs(ckmpm_scene* s, ModelHost& m, const float* x, const float* v) {
  cudaError_t e = cudaSetDevice(s->desc.device);
  if (e != cudaSuccess) return e;
  const bool track = m.mat.kind == kMixedKind || (s->desc.flags & CKMPM_FLAG_TRACK_IDS) != 0;
  Carve size;
  io_layout(m, track, size);
  e = cudaMalloc(&m.io, size.off);
  if (e != cudaSuccess) {
    m.io = nullptr;
    return e;
  }
  Carve place{m.io, 0};
  io_layout(m, track, place);
  if (!m.ev_copied) e = cudaEventCreateWithFlags(&m.ev_copied, cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m.ox, x, sizeof(float) * 3 * static_cast<size_t>(m.n), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m.ov, v, sizeof(float) * 3 * static_cast<size_t>(m.nv), cudaMemcpyHostToDevice, s->stream);
  // The state arena is made while the copies run (cudaMalloc does not wait for
  // the device): on the sand column it overlapped ~0.3 ms of allocation with
  // the 40 MB upload.
  const size_t nallocs = s->allocs.size();
  if (e == cudaSuccess) e = alloc_state(s, m);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(s->stream);
    cudaFree(m.io);
    m.io = nullptr;
    if (m.ev_copied) cudaEventDestroy(m.ev_copied);
    m.ev_copied = nullptr;
    while (s->allocs.size() > nallocs) {
      cudaFree(s->allocs.back().first);
      s->allocs.pop_back();
    }
  }
  return e;
}

extern "C" {

const char* ckmpm_version(void) { return kVersion; }

ckmpm_status ckmpm_create(const ckmpm_scene_desc* desc, ckmpm_scene** out) { return create_impl(desc, 1, out); }

ckmpm_status ckmpm_create_batch(const ckmpm_scene_desc* desc, uint32_t nscenes, ckmpm_scene** out) {
  return create_impl(desc, nscenes, out);
}

ckmpm_status ckmpm_add_batch(ckmpm_scene* s, uint32_t nscenes, const ckmpm_batch_scene* scenes, const float* x,
                             const float* v) {
  if (!s || !scenes || !x || !v) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (s->setup_done) return fail(s, CKMPM_ERR_INVALID, "scenes must be added before ckmpm_setup");
  if (!s->models.empty()) return fail(s, CKMPM_ERR_INVALID, "a batch holds exactly one ckmpm_add_batch call");
  if (nscenes != s->nstack) return fail(s, CKMPM_ERR_INVALID, "nscenes differs from ckmpm_create_batch");
  ModelHost m;
  m.mat.kind = kMixedKind;
  m.smat.resize(nscenes);
  m.skind.resize(nscenes);
  m.sstart.assign(nscenes + 1, 0u);
  uint64_t total = 0;
  float lightest = 0.f;
  for (uint32_t i = 0; i < nscenes; ++i) {
    const ckmpm_batch_scene& b = scenes[i];
    const int k = b.material.kind;
    std::string why;
    if (!valid_material(b.material, &why)) return fail(s, CKMPM_ERR_INVALID, why + " (scene " + std::to_string(i) + ")");
    if (!(b.mass > 0.f) || !(b.volume > 0.f))
      return fail(s, CKMPM_ERR_INVALID, "mass and volume must be positive (scene " + std::to_string(i) + ")");
    SceneMat& sm = m.smat[i];
    sm.kind = k;
    for (int j = 0; j < kMaterialParams; ++j) sm.p[j] = b.material.p[j];
    sm.vol_over_mass = b.volume / b.mass;
    sm.unit = b.mass * kFixInvScale;
    sm.aux0 = initial_aux(b.material);
    m.skind[i] = k;
    m.sstart[i] = static_cast<uint32_t>(total);
    total += b.n;
    lightest = (i == 0) ? b.mass : std::min(lightest, b.mass);
  }
  if (total == 0 || total > 0xFFFFFFF0ull) return fail(s, CKMPM_ERR_INVALID, "batch particle count out of range");
  m.sstart[nscenes] = static_cast<uint32_t>(total);
  m.n = static_cast<uint32_t>(total);
  m.nv = m.n;
  m.mass = lightest;  // only the adaptive-dt mass floor reads it for a batch
  m.vol = 1.f;
  CK_CUDA(s, stage_inputs(s, m, x, v));
  s->models.push_back(std::move(m));
  return CKMPM_OK;
}

ckmpm_status ckmpm_set_tuning(ckmpm_scene* s, const ckmpm_tuning* t) {
  if (!s || !t) return fail(s, CKMPM_ERR_INVALID, "null argument");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  return apply_tuning(s, *t);
}

ckmpm_status ckmpm_set_reorder_interval(ckmpm_scene* s, uint32_t substeps) {
  if (!s) return fail(s, CKMPM_ERR_INVALID, "null argument");
  s->reorder_every = substeps;
  return CKMPM_OK;
}

ckmpm_status ckmpm_get_tuning(ckmpm_scene* s, ckmpm_tuning* t, uint32_t* max_ctas_per_sm2) {
  if (!s || !t) return fail(s, CKMPM_ERR_INVALID, "null argument");
  *t = s->tune;
  if (max_ctas_per_sm2) {
    max_ctas_per_sm2[0] = static_cast<uint32_t>(s->occ[0]);
    max_ctas_per_sm2[1] = static_cast<uint32_t>(s->occ[1]);
  }
  return CKMPM_OK;
}

ckmpm_status ckmpm_checkpoint_bytes(ckmpm_scene* s, uint64_t* bytes) {
  if (!s || !bytes) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  *bytes = checkpoint_bytes(s);
  return CKMPM_OK;
}

ckmpm_status ckmpm_checkpoint_save(ckmpm_scene* s, void* device_dst) {
  if (!s || !device_dst) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  CK_CUDA(s, checkpoint_copy(s, static_cast<unsigned char*>(device_dst), true));
  return CKMPM_OK;
}

ckmpm_status ckmpm_checkpoint_restore(ckmpm_scene* s, const void* device_src) {
  if (!s || !device_src) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  CK_CUDA(s, checkpoint_copy(s, static_cast<unsigned char*>(const_cast<void*>(device_src)), false));
  Scalars h{};
  CK_CUDA(s, cudaMemcpyAsync(&h, s->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  s->host_step = static_cast<uint64_t>(h.step);
  return CKMPM_OK;
}

const char* ckmpm_last_error(const ckmpm_scene* s) { return s ? s->err.c_str() : g_create_error.c_str(); }

ckmpm_status ckmpm_add_model(ckmpm_scene* s, const ckmpm_material* material, uint32_t n, const float* x,
                             const float* v, uint32_t nv, float mass, float volume, int32_t* model_index) {
  if (!s || !material || !x || !v) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (s->setup_done) return fail(s, CKMPM_ERR_INVALID, "models must be added before ckmpm_setup");
  if (n == 0) return fail(s, CKMPM_ERR_INVALID, "empty model");
  if (nv != 1 && nv != n) return fail(s, CKMPM_ERR_INVALID, "nv must be 1 or n");
  std::string why;
  if (!valid_material(*material, &why)) return fail(s, CKMPM_ERR_INVALID, why);
  if (!(mass > 0.f) || !(volume > 0.f)) return fail(s, CKMPM_ERR_INVALID, "mass and volume must be positive");
  ModelHost m;
  m.mat = *material;
  m.mass = mass;
  m.vol = volume;
  m.n = n;
  m.nv = nv;
  CK_CUDA(s, stage_inputs(s, m, x, v));
  s->models.push_back(std::move(m));
  if (model_index) *model_index = static_cast<int32_t>(s->models.size()) - 1;
  return CKMPM_OK;
}

// The previous-step lists bl[list ^ 1] as the identity over bl[list]: the same
// blocks, every particle staying in its block at its own position, so the next
// substep (whose list is bl[list]) reads the state in bl[list]'s layout
// (include/mpm_algorithm.cuh:950-964 InitializeAdvectionBucket).
static cudaError_t identity_previous_lists(ckmpm_scene* s, ModelDev& d, int list) {
  const BlockListDev& a = d.bl[list];
  const BlockListDev& b = d.bl[list ^ 1];
  const uint32_t nbd = s->sc.nblocks_domain;
  cudaError_t e = cudaMemcpyAsync(b.table, a.table, sizeof(int32_t) * nbd, cudaMemcpyDeviceToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b.start, a.start, sizeof(uint32_t) * d.cap_slots, cudaMemcpyDeviceToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b.count, a.count, sizeof(uint32_t) * d.cap_slots, cudaMemcpyDeviceToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b.keys, a.keys, sizeof(int4) * d.cap_slots, cudaMemcpyDeviceToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b.nblocks, a.nblocks, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b.nparticles, a.nparticles, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s->stream);
  if (e != cudaSuccess) return e;
  setup_identity_kernel<<<s->sm_count * 4, 256, 0, s->stream>>>(a, b);
  return cudaGetLastError();
}

// Re-layout of every model's particles before the next substep
// (reorder_gather_kernel): gather into the free state buffer in the setup
// order, copy it back, make the previous-step lists the identity.
static cudaError_t enqueue_reorder(ckmpm_scene* s) {
  const int list = static_cast<int>(s->host_step & 1);
  for (auto& m : s->models) {
    ModelDev& d = m.dev;
    reorder_gather_kernel<256><<<s->sm_count * 4, 256, 0, s->stream>>>(s->sc, d, list, s->scal);
    cudaError_t e = cudaGetLastError();
    const StateDev& to = d.st[list];
    const StateDev& from = d.st[list ^ 1];
    const size_t bytes = sizeof(float) * d.cap_particles;
    auto copy = [&](void* dst, const void* src) {
      if (e == cudaSuccess && dst) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s->stream);
    };
    for (int a = 0; a < 3; ++a) copy(to.x[a], from.x[a]);
    for (int k = 0; k < 9; ++k) copy(to.F[k], from.F[k]);
    copy(to.aux, from.aux);
    for (int k = 0; k < 9; ++k) copy(to.Q[k], from.Q[k]);
    copy(to.id, from.id);
    if (e == cudaSuccess) e = identity_previous_lists(s, d, list);
    if (e != cudaSuccess) return e;
  }
  s->last_reorder = s->host_step;
  return cudaSuccess;
}

// Whether the re-layout is due before the next substep, and whether one falls
// strictly inside the next k substeps (a chunk graph must not cover it).
static bool reorder_due(const ckmpm_scene* s) {
  return s->reorder_every && s->host_step > 0 && s->host_step % s->reorder_every == 0 &&
         s->last_reorder != s->host_step;
}
static bool reorder_inside(const ckmpm_scene* s, uint32_t k) {
  if (!s->reorder_every) return false;
  const uint64_t next = (s->host_step / s->reorder_every + 1) * s->reorder_every;
  return next < s->host_step + k;
}

ckmpm_status ckmpm_setup(ckmpm_scene* s) {
  if (!s) return fail(s, CKMPM_ERR_INVALID, "null scene");
  if (s->setup_done) return fail(s, CKMPM_ERR_INVALID, "setup already done");
  if (s->models.empty()) return fail(s, CKMPM_ERR_INVALID, "no models");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  const uint32_t nbd = s->sc.nblocks_domain;
  // The grid's fixed-point unit: 2^-36 of the heaviest model's particle mass;
  // lighter models' sums are rescaled when they are added.  A batch uses each
  // scene's own mass (one model per scene).
  float heaviest = 0.f;
  for (const auto& m : s->models) heaviest = std::max(heaviest, m.mass);
  s->sc.grid_unit = heaviest * kFixInvScale;
  for (auto& m : s->models) {
    ModelDev& d = m.dev;
    d.flush_ratio = static_cast<double>(m.mass) / static_cast<double>(heaviest);
    const uint32_t n = m.n;
    const bool batch = m.mat.kind == kMixedKind;
    // A batch always tracks ids: they map each particle back to its scene.
    const bool track = batch || (s->desc.flags & CKMPM_FLAG_TRACK_IDS) != 0;
    // cap_particles, cap_slots, ntiles and the state arrays were placed when
    // the model was added (alloc_state).
    d.max_per_block = s->desc.max_particles_per_block;
    d.track_ids = track ? 1 : 0;
    d.mat.kind = m.mat.kind;
    for (int k = 0; k < kMaterialParams; ++k) d.mat.p[k] = m.mat.p[k];
    d.mass = m.mass;
    d.vol = m.vol;
    for (int b = 0; b < 2; ++b) {
      CK_CUDA(s, cudaMemsetAsync(d.bl[b].nblocks, 0, sizeof(uint32_t), s->stream));
      CK_CUDA(s, cudaMemsetAsync(d.bl[b].nparticles, 0, sizeof(uint32_t), s->stream));
    }
    CK_CUDA(s, cudaMemsetAsync(d.dense_total, 0, sizeof(uint32_t) * nbd, s->stream));
    CK_CUDA(s, cudaMemsetAsync(d.ticket, 0, sizeof(uint32_t), s->stream));
    if (batch) {
      CK_CUDA(s, cudaMemcpyAsync(const_cast<SceneMat*>(d.smat), m.smat.data(), sizeof(SceneMat) * m.smat.size(),
                                 cudaMemcpyHostToDevice, s->stream));
      CK_CUDA(s, cudaMemcpyAsync(const_cast<uint32_t*>(d.sstart), m.sstart.data(), sizeof(uint32_t) * m.sstart.size(),
                                 cudaMemcpyHostToDevice, s->stream));
    }

    // Bin, compact into the colour-major block list, place every particle in
    // its block's range and order each range (by input index, then interleaved
    // across the block's cells, setup_order_kernel); the inputs and these
    // arrays live in the model's I/O arena.  Nothing here waits for the
    // device: kernels that depend on the binned count read it on the device.
    uint32_t* flat = sort_array(m, 0);
    uint32_t* cursor = sort_array(m, 1);
    uint32_t* perm = sort_array(m, 2);
    setup_bin_kernel<<<(n + 255) / 256, 256, 0, s->stream>>>(s->sc, n, m.ox, d.sstart, flat, d.dense_total);
    CK_CUDA(s, launch_compact(s, m, d.bl[0]));
    CK_CUDA(s, cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * d.cap_slots, s->stream));
    setup_place_kernel<<<(n + 255) / 256, 256, 0, s->stream>>>(n, flat, d.bl[0], cursor, perm);
    setup_order_kernel<256><<<s->sm_count * 4, 256, 0, s->stream>>>(s->sc, d.bl[0], m.ox, perm, s->scal);
    const float aux0 = initial_aux(m.mat);
    setup_gather_kernel<<<(n + 255) / 256, 256, 0, s->stream>>>(
        d, s->nstack, n, perm, m.ox, m.ov, m.nv, aux0,
        (s->sc.rigid && m.mat.kind == CKMPM_VON_MISES) ? s->rigid_count : 0u, d.bl[0].nparticles);
    // Identity previous-step structures in list 1.
    CK_CUDA(s, identity_previous_lists(s, d, 0));
    // Particles outside the domain are dropped at binning and counted.
    count_lost_kernel<<<1, 32, 0, s->stream>>>(s->scal, n, d.bl[0].nparticles);
    CK_CUDA(s, cudaGetLastError());
  }
  // Initial grid: every model deposits mass and momentum into grid[0], epoch 0;
  // then the blocks substep 0 deposits into are zeroed in grid[1] (epoch 1).
  CK_CUDA(s, launch_zero(s, 0, 0, 0));
  for (auto& m : s->models) {
    CK_CUDA(s, cudaMemsetAsync(m.dev.ticket, 0, sizeof(uint32_t), s->stream));
    rasterize_kernel<kFusedThreads><<<s->fused_ctas, kFusedThreads, kSmemFused, s->stream>>>(s->sc, m.dev, s->grid,
                                                                                             s->scal);
    CK_CUDA(s, cudaGetLastError());
    CK_CUDA(s, cudaMemsetAsync(m.dev.ticket, 0, sizeof(uint32_t), s->stream));
  }
  CK_CUDA(s, launch_zero(s, 0, 1, 1));
  // The scalars were zeroed at creation; setup's kernels may have raised status
  // bits in them, which ckmpm_setup then reports.
  finish_setup_kernel<<<1, 32, 0, s->stream>>>(s->scal, 0u, s->rigid_v[0], s->rigid_v[1], s->rigid_v[2]);
  CK_CUDA(s, cudaGetLastError());
  // The one wait of setup: the status word and each model's binned count.
  std::vector<uint32_t> binned(s->models.size(), 0u);
  for (size_t i = 0; i < s->models.size(); ++i)
    CK_CUDA(s, cudaMemcpyAsync(&binned[i], s->models[i].dev.bl[0].nparticles, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               s->stream));
  Scalars r{};
  CK_CUDA(s, cudaMemcpyAsync(&r, s->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  for (size_t i = 0; i < s->models.size(); ++i) s->models[i].n_valid = binned[i];
  s->setup_done = true;
  s->host_step = 0;
  s->n_state_allocs = s->allocs.size();
  return status_from(s, r);
}

ckmpm_status ckmpm_set_boundary_field(ckmpm_scene* s, const uint8_t* rule, const float* param) {
  if (!s || !rule) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (s->desc.boundary != CKMPM_BOUNDARY_FIELD || !s->sc.brule)
    return fail(s, CKMPM_ERR_INVALID, "the scene's boundary kind is not CKMPM_BOUNDARY_FIELD");
  const size_t cells = static_cast<size_t>(s->desc.domain_blocks[0]) * s->desc.domain_blocks[1] *
                       s->desc.domain_blocks[2] * 64;
  bool needs_param = false;
  for (size_t c = 0; c < cells; ++c) {
    if (rule[c] > CKMPM_CELL_SEPARATE) return fail(s, CKMPM_ERR_INVALID, "unknown cell rule");
    needs_param |= rule[c] >= CKMPM_CELL_SLIP;
  }
  if (needs_param && !param) return fail(s, CKMPM_ERR_INVALID, "SLIP, VELOCITY and SEPARATE cells need param");
  if (param)
    for (size_t k = 0; k < 3 * cells; ++k)
      if (!std::isfinite(param[k])) return fail(s, CKMPM_ERR_INVALID, "boundary parameters must be finite");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  // Stream-ordered: substeps already enqueued keep the old field.  Pageable
  // sources are staged before the calls return.
  CK_CUDA(s, cudaMemcpyAsync(const_cast<uint8_t*>(s->sc.brule), rule, cells, cudaMemcpyHostToDevice, s->stream));
  if (param)
    CK_CUDA(s, cudaMemcpyAsync(const_cast<float*>(s->sc.bparam), param, sizeof(float) * 3 * cells,
                               cudaMemcpyHostToDevice, s->stream));
  return CKMPM_OK;
}

ckmpm_status ckmpm_set_rigid(ckmpm_scene* s, uint32_t rigid_count, const float* velocity) {
  if (!s || !velocity) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (s->setup_done) return fail(s, CKMPM_ERR_INVALID, "rigid particles are set before ckmpm_setup");
  if (s->nstack > 1) return fail(s, CKMPM_ERR_INVALID, "a batch has no rigid particles");
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(velocity[a])) return fail(s, CKMPM_ERR_INVALID, "rigid velocity must be finite");
  s->sc.rigid = 1;
  s->rigid_count = rigid_count;
  for (int a = 0; a < 3; ++a) s->rigid_v[a] = velocity[a];
  return CKMPM_OK;
}

ckmpm_status ckmpm_set_rigid_velocity(ckmpm_scene* s, const float* velocity) {
  if (!s || !velocity) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (!s->sc.rigid) return fail(s, CKMPM_ERR_INVALID, "rigid particles are off (ckmpm_set_rigid)");
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(velocity[a])) return fail(s, CKMPM_ERR_INVALID, "rigid velocity must be finite");
  for (int a = 0; a < 3; ++a) s->rigid_v[a] = velocity[a];
  if (!s->setup_done) return CKMPM_OK;
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  // Stream-ordered: substeps already enqueued keep the old velocity.  The
  // pageable source is staged before the call returns.
  CK_CUDA(s, cudaMemcpyAsync(s->scal->rigid_v, s->rigid_v, sizeof(s->rigid_v), cudaMemcpyHostToDevice, s->stream));
  return CKMPM_OK;
}

ckmpm_status ckmpm_set_stream(ckmpm_scene* s, void* cuda_stream) {
  if (!s) return fail(s, CKMPM_ERR_INVALID, "null scene");
  s->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : s->own_stream;
  return CKMPM_OK;
}

ckmpm_status ckmpm_step_async(ckmpm_scene* s, uint32_t nsteps, float dt) {
  if (!s || !s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (!(dt >= 0.f)) return fail(s, CKMPM_ERR_INVALID, "dt must be non-negative");
  if (nsteps == 0) return CKMPM_OK;
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  set_next_dt_kernel<<<1, 32, 0, s->stream>>>(s->scal, dt);
  CK_CUDA(s, cudaGetLastError());
  // The parity of the substep counter decides which block list each
  // compaction writes.  The device counter only moves through these launches,
  // so the host mirror is exact; chunk graphs are captured at even parity.
  uint32_t done = 0;
  while (done < nsteps) {
    if (reorder_due(s)) CK_CUDA(s, enqueue_reorder(s));
    const int parity = static_cast<int>(s->host_step & 1);
    const uint32_t chunk = s->tune.graph_chunk;
    if (parity == 0 && nsteps - done >= chunk && !reorder_inside(s, chunk)) {
      if (!s->graph_chunk) CK_CUDA(s, build_graph(s, static_cast<int>(chunk), 0, &s->graph_chunk));
      CK_CUDA(s, cudaGraphLaunch(s->graph_chunk, s->stream));
      done += chunk;
      s->host_step += chunk;
    } else {
      CK_CUDA(s, enqueue_substep(s, parity));
      ++done;
      ++s->host_step;
    }
  }
  return CKMPM_OK;
}

ckmpm_status ckmpm_status_check(ckmpm_scene* s) {
  if (!s) return fail(s, CKMPM_ERR_INVALID, "null scene");
  Scalars h{};
  CK_CUDA(s, cudaMemcpyAsync(&h, s->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  return status_from(s, h);
}

ckmpm_status ckmpm_step(ckmpm_scene* s, uint32_t nsteps, float dt) {
  ckmpm_status st = ckmpm_step_async(s, nsteps, dt);
  if (st != CKMPM_OK) return st;
  return ckmpm_status_check(s);
}

ckmpm_status ckmpm_step_adaptive(ckmpm_scene* s, uint32_t nsteps, float dt_max, float cfl, double frame_time,
                                 double* elapsed) {
  if (!s || !s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (!(dt_max > 0.f) || !(cfl > 0.f) || !(frame_time >= 0.0))
    return fail(s, CKMPM_ERR_INVALID, "dt_max and cfl must be positive, frame_time non-negative");
  if (s->nstack > 1) return fail(s, CKMPM_ERR_INVALID, "a batch steps with a fixed dt (ckmpm_step)");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  Scalars h{};
  CK_CUDA(s, cudaMemcpyAsync(&h, s->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  // frame_time == 0 continues the frame an earlier call opened (a caller that
  // steps one substep at a time, e.g. to record per-substep diagnostics).
  const double t0 = h.time, t_end = frame_time > 0.0 ? h.time + frame_time : h.frame_end;
  if (frame_time > 0.0) set_frame_end_kernel<<<1, 32, 0, s->stream>>>(s->scal, frame_time);
  const int maxv_ctas = s->sm_count * 8;
  float mass_floor = 0.f;
  for (const auto& m : s->models) mass_floor = (mass_floor == 0.f) ? m.mass : std::min(mass_floor, m.mass);
  mass_floor *= 1.52587890625e-05f;  // 2^-16
  uint32_t taken = 0;
  // Each substep advances by at most dt_max, so floor(remaining / dt_max)
  // substeps never pass the frame end; the last one is clipped to it on the
  // device, as the reference's frame loop does (include/mpm_engine.cuh:514-552).
  for (;;) {
    const double remaining = t_end - h.time;
    if (!(remaining > 0.0) || taken >= nsteps) break;
    uint32_t k = static_cast<uint32_t>(remaining / static_cast<double>(dt_max));
    k = std::max<uint32_t>(1u, std::min<uint32_t>(k, nsteps - taken));
    for (uint32_t i = 0; i < k; ++i) {
      if (reorder_due(s)) CK_CUDA(s, enqueue_reorder(s));
      const int parity = static_cast<int>(s->host_step & 1);
      grid_maxv_kernel<<<maxv_ctas, 256, 0, s->stream>>>(s->sc, s->grid, s->scal, mass_floor);
      adaptive_dt_kernel<<<1, 32, 0, s->stream>>>(s->scal, s->sc.dx, cfl, dt_max);
      CK_CUDA(s, enqueue_substep(s, parity));
      ++s->host_step;
    }
    taken += k;
    CK_CUDA(s, cudaMemcpyAsync(&h, s->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
    CK_CUDA(s, cudaStreamSynchronize(s->stream));
    ckmpm_status st = status_from(s, h);
    if (st != CKMPM_OK) return st;
  }
  if (elapsed) *elapsed = h.time - t0;
  return CKMPM_OK;
}

ckmpm_status ckmpm_get_count(ckmpm_scene* s, int32_t model, uint32_t* n_live) {
  if (!s || !n_live) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (model < 0 || model >= static_cast<int32_t>(s->models.size())) return fail(s, CKMPM_ERR_NOT_FOUND, "no such model");
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  const BlockListDev& cur = s->models[model].dev.bl[s->host_step & 1];
  CK_CUDA(s, cudaMemcpy(n_live, cur.nparticles, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return CKMPM_OK;
}

// Export buffers of one model: part of its I/O arena (ckmpm_add_model).
static cudaError_t ensure_export_buffers(ckmpm_scene*, ModelHost& m) {
  return (m.ox && m.ov && m.oF && m.oaux && m.oid && (!m.dev.track_ids || (m.oflag && m.opos && m.oscan)))
             ? cudaSuccess
             : cudaErrorInvalidValue;
}

// Enqueues the gather of the requested per-particle arrays into the model's
// export buffers (input order when ids are tracked).  n_upper bounds the live
// count; n_dev, when given, is the device copy of it.
static cudaError_t enqueue_export(ckmpm_scene* s, ModelHost& m, bool x, bool v, bool F, bool aux, bool id,
                                  uint32_t n_upper, const uint32_t* n_dev) {
  const size_t cap_p = m.dev.cap_particles;
  const dim3 pg(s->sm_count * 4), pb(kProbeThreads);
  const uint32_t* dest = nullptr;
  cudaError_t e;
  if (m.copy_pending && (e = cudaStreamWaitEvent(s->stream, m.ev_copied, 0)) != cudaSuccess) return e;
  if (m.dev.track_ids) {
    // ids in block order, then the position of each live id in input order
    probe_kernel<kProbeThreads><<<pg, pb, kSmemVTile, s->stream>>>(s->sc, m.dev, s->grid, s->scal, nullptr, nullptr,
                                                                 nullptr, nullptr, m.oid, nullptr);
    if ((e = cudaMemsetAsync(m.oflag, 0, sizeof(uint32_t) * cap_p, s->stream)) != cudaSuccess) return e;
    if (n_upper)
      mark_ids_kernel<<<(n_upper + 255) / 256, 256, 0, s->stream>>>(n_upper, m.oid, m.oflag,
                                                                    static_cast<uint32_t>(cap_p), n_dev);
    const uint32_t ntiles = scan_tiles(static_cast<uint32_t>(cap_p));
    scan_reduce_kernel<<<ntiles, kScanThreads, 0, s->stream>>>(m.oflag, static_cast<uint32_t>(cap_p), m.oscan);
    scan_sums_kernel<<<1, kScanThreads, 0, s->stream>>>(m.oscan, ntiles);
    scan_apply_kernel<<<ntiles, kScanThreads, 0, s->stream>>>(m.oflag, static_cast<uint32_t>(cap_p), m.oscan, m.opos);
    dest = m.opos;
  }
  probe_kernel<kProbeThreads><<<pg, pb, kSmemVTile, s->stream>>>(s->sc, m.dev, s->grid, s->scal, x ? m.ox : nullptr,
                                                               v ? m.ov : nullptr, F ? m.oF : nullptr,
                                                               aux ? m.oaux : nullptr, id ? m.oid : nullptr, dest);
  return cudaGetLastError();
}

ckmpm_status ckmpm_get_state(ckmpm_scene* s, int32_t model, float* x, float* v, float* F, float* aux, uint32_t* id,
                             uint32_t cap, uint32_t* n_out) {
  if (!s) return fail(s, CKMPM_ERR_INVALID, "null scene");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (model < 0 || model >= static_cast<int32_t>(s->models.size())) return fail(s, CKMPM_ERR_NOT_FOUND, "no such model");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  ModelHost& m = s->models[model];
  uint32_t n = 0;
  ckmpm_status st = ckmpm_get_count(s, model, &n);
  if (st != CKMPM_OK) return st;
  if (n_out) *n_out = n;
  if (cap < n) return fail(s, CKMPM_ERR_NOT_FOUND, "output capacity too small");
  if (n == 0) return CKMPM_OK;
  CK_CUDA(s, ensure_export_buffers(s, m));
  CK_CUDA(s, enqueue_export(s, m, x, v, F, aux, id, n, nullptr));
  if (x) CK_CUDA(s, cudaMemcpyAsync(x, m.ox, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s->stream));
  if (v) CK_CUDA(s, cudaMemcpyAsync(v, m.ov, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s->stream));
  if (F) CK_CUDA(s, cudaMemcpyAsync(F, m.oF, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost, s->stream));
  if (aux) CK_CUDA(s, cudaMemcpyAsync(aux, m.oaux, sizeof(float) * n, cudaMemcpyDeviceToHost, s->stream));
  if (id) CK_CUDA(s, cudaMemcpyAsync(id, m.oid, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s->stream));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  return CKMPM_OK;
}

ckmpm_status ckmpm_export_positions_async(ckmpm_scene* s, int32_t model, float* x, uint32_t cap) {
  if (!s || !x) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (model < 0 || model >= static_cast<int32_t>(s->models.size())) return fail(s, CKMPM_ERR_NOT_FOUND, "no such model");
  ModelHost& m = s->models[model];
  // Live particles never exceed those binned at setup, nor the id range.
  const uint32_t n_upper = m.n_valid;
  if (cap < n_upper) return fail(s, CKMPM_ERR_NOT_FOUND, "output capacity too small");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  CK_CUDA(s, ensure_export_buffers(s, m));
  const uint32_t* n_dev = m.dev.bl[s->host_step & 1].nparticles;
  CK_CUDA(s, enqueue_export(s, m, true, false, false, false, false, n_upper, n_dev));
  CK_CUDA(s, cudaEventRecord(s->ev_probe, s->stream));
  CK_CUDA(s, cudaStreamWaitEvent(s->copy_stream, s->ev_probe, 0));
  CK_CUDA(s, cudaMemcpyAsync(s->export_count, n_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->copy_stream));
  if (n_upper)
    CK_CUDA(s, cudaMemcpyAsync(x, m.ox, sizeof(float) * 3 * n_upper, cudaMemcpyDeviceToHost, s->copy_stream));
  CK_CUDA(s, cudaEventRecord(m.ev_copied, s->copy_stream));
  CK_CUDA(s, cudaEventRecord(s->ev_copy, s->copy_stream));
  m.copy_pending = true;
  s->export_pending = true;
  return CKMPM_OK;
}

ckmpm_status ckmpm_export_wait(ckmpm_scene* s, uint32_t* n_out) {
  if (!s) return fail(s, CKMPM_ERR_INVALID, "null scene");
  if (!s->export_pending) {
    if (n_out) *n_out = s->export_count ? *s->export_count : 0u;
    return CKMPM_OK;
  }
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  CK_CUDA(s, cudaEventSynchronize(s->ev_copy));  // the copy stream runs in order: every export is done
  s->export_pending = false;
  for (auto& m : s->models) m.copy_pending = false;
  if (n_out) *n_out = *s->export_count;
  return CKMPM_OK;
}

ckmpm_status ckmpm_get_blocks(ckmpm_scene* s, int32_t model, int32_t which, int32_t* keys, uint32_t* counts,
                              uint32_t cap, uint32_t* n_out) {
  return ckmpm_get_blocks_in(s, 0, model, which, keys, counts, cap, n_out);
}

ckmpm_status ckmpm_get_blocks_in(ckmpm_scene* s, uint32_t scene, int32_t model, int32_t which, int32_t* keys,
                                 uint32_t* counts, uint32_t cap, uint32_t* n_out) {
  if (!s) return fail(s, CKMPM_ERR_INVALID, "null scene");
  if (scene >= s->nstack) return fail(s, CKMPM_ERR_NOT_FOUND, "no such scene in the batch");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (which < 0 || which > 2) return fail(s, CKMPM_ERR_INVALID, "which must be 0, 1 or 2");
  if (model >= static_cast<int32_t>(s->models.size())) return fail(s, CKMPM_ERR_NOT_FOUND, "no such model");
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  const uint64_t step = s->host_step;
  std::map<std::tuple<int, int, int>, uint32_t> set;
  for (int32_t mi = 0; mi < static_cast<int32_t>(s->models.size()); ++mi) {
    if (model >= 0 && mi != model) continue;
    const BlockListDev& cur = s->models[mi].dev.bl[step & 1];
    uint32_t nb = 0;
    CK_CUDA(s, cudaMemcpy(&nb, cur.nblocks, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    std::vector<int4> hk(nb);
    std::vector<uint32_t> hc(nb);
    if (nb) {
      CK_CUDA(s, cudaMemcpy(hk.data(), cur.keys, sizeof(int4) * nb, cudaMemcpyDeviceToHost));
      CK_CUDA(s, cudaMemcpy(hc.data(), cur.count, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost));
    }
    for (uint32_t i = 0; i < nb; ++i)
      if (static_cast<uint32_t>(hk[i].w) == scene) set[std::make_tuple(hk[i].x, hk[i].y, hk[i].z)] += hc[i];
    if (step == 0 && nb) {
      // Right after setup the reference's partition also holds the blocks of
      // each particle's cell on the +dx/4 grid, (int(x/dx - 1/4) - 2) / 4
      // (ActivateBlocksWithParticles inserts both staggered grids' blocks,
      // include/mpm_algorithm.cuh:713-736); they hold no particles.  The
      // first rebinning keeps only blocks with particles, as here.
      std::vector<uint32_t> hs(nb);
      CK_CUDA(s, cudaMemcpy(hs.data(), cur.start, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost));
      const StateDev& st = s->models[mi].dev.st[0];
      const uint32_t np = s->models[mi].n_valid;
      std::vector<float> hx[3];
      for (int a = 0; a < 3; ++a) {
        hx[a].resize(np);
        if (np) CK_CUDA(s, cudaMemcpy(hx[a].data(), st.x[a], sizeof(float) * np, cudaMemcpyDeviceToHost));
      }
      const float inv_dx = s->sc.inv_dx;
      for (uint32_t i = 0; i < nb; ++i) {
        if (static_cast<uint32_t>(hk[i].w) != scene) continue;
        for (uint32_t p = hs[i]; p < hs[i] + hc[i] && p < np; ++p) {
          int b[3];
          for (int a = 0; a < 3; ++a) b[a] = (static_cast<int>(std::fma(hx[a][p], inv_dx, -0.25f)) - 2) / 4;
          if (b[0] >= 0 && b[1] >= 0 && b[2] >= 0 && b[0] < s->sc.dims[0] && b[1] < s->sc.dims[1] &&
              b[2] < s->sc.dims[2])
            set.emplace(std::make_tuple(b[0], b[1], b[2]), 0u);
        }
      }
    }
  }
  if (which >= 1) {
    const int lo = which == 1 ? 0 : -1;
    std::map<std::tuple<int, int, int>, uint32_t> ext = set;
    for (auto& kv : set) {
      const int bx = std::get<0>(kv.first), by = std::get<1>(kv.first), bz = std::get<2>(kv.first);
      for (int i = lo; i <= 1; ++i)
        for (int j = lo; j <= 1; ++j)
          for (int k = lo; k <= 1; ++k) {
            const int x = bx + i, y = by + j, z = bz + k;
            if (x < 0 || y < 0 || z < 0 || x >= s->sc.dims[0] || y >= s->sc.dims[1] || z >= s->sc.dims[2]) continue;
            ext.emplace(std::make_tuple(x, y, z), 0u);
          }
    }
    set.swap(ext);
  }
  const uint32_t n = static_cast<uint32_t>(set.size());
  if (n_out) *n_out = n;
  if (cap < n) return fail(s, CKMPM_ERR_NOT_FOUND, "output capacity too small");
  uint32_t i = 0;
  for (auto& kv : set) {
    if (keys) {
      keys[3 * i] = std::get<0>(kv.first);
      keys[3 * i + 1] = std::get<1>(kv.first);
      keys[3 * i + 2] = std::get<2>(kv.first);
    }
    if (counts) counts[i] = kv.second;
    ++i;
  }
  return CKMPM_OK;
}

ckmpm_status ckmpm_autotune(ckmpm_scene* s, uint32_t probe_steps, float dt, ckmpm_tuning* results, uint32_t cap,
                            uint32_t* n_results, ckmpm_tuning* best) {
  if (!s || !best) return fail(s, CKMPM_ERR_INVALID, "null argument");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (probe_steps < 2 || probe_steps > 4096) return fail(s, CKMPM_ERR_INVALID, "probe_steps must be 2..4096");
  if (!(dt >= 0.f)) return fail(s, CKMPM_ERR_INVALID, "dt must be non-negative");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  // The probes advance the simulation; the state is saved first and put back
  // after every candidate, so tuning leaves the scene exactly as it found it.
  const size_t bytes = checkpoint_bytes(s);
  void* saved = nullptr;
  CK_CUDA(s, cudaMalloc(&saved, bytes));
  struct Guard {
    void* p;
    ~Guard() { cudaFree(p); }
  } guard{saved};
  CK_CUDA(s, checkpoint_copy(s, static_cast<unsigned char*>(saved), true));
  const ckmpm_tuning before = s->tune;
  std::vector<ckmpm_tuning> cands;
  for (uint32_t nt : {256u, 192u, 128u, 1024u}) {
    const int occ = s->occ[shape_index(nt)];
    for (int c = occ; c >= 1; --c)
      for (uint32_t chunk : {8u, 32u}) cands.push_back(ckmpm_tuning{nt, static_cast<uint32_t>(c), chunk, 0.f});
  }
  cudaEvent_t e0, e1;
  CK_CUDA(s, cudaEventCreate(&e0));
  CK_CUDA(s, cudaEventCreate(&e1));
  ckmpm_status result = CKMPM_OK;
  for (auto& c : cands) {
    ckmpm_status st = CKMPM_OK;
    if ((st = ckmpm_checkpoint_restore(s, saved)) != CKMPM_OK || (st = apply_tuning(s, c)) != CKMPM_OK ||
        (st = ckmpm_step_async(s, c.graph_chunk, dt)) != CKMPM_OK) {  // warm-up; captures this shape's graph
      result = st;
      break;
    }
    const uint32_t k = ((probe_steps + c.graph_chunk - 1) / c.graph_chunk) * c.graph_chunk;
    cudaEventRecord(e0, s->stream);
    st = ckmpm_step_async(s, k, dt);
    cudaEventRecord(e1, s->stream);
    if (st == CKMPM_OK) st = ckmpm_status_check(s);
    if (st != CKMPM_OK) {
      result = st;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    c.probe_ms = ms / static_cast<float>(k);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ckmpm_status rs = ckmpm_checkpoint_restore(s, saved);
  if (result != CKMPM_OK) {
    apply_tuning(s, before);
    return result;
  }
  if (rs != CKMPM_OK) return rs;
  const ckmpm_tuning* pick = &cands[0];
  for (const auto& c : cands)
    if (c.probe_ms < pick->probe_ms) pick = &c;
  *best = *pick;
  if (n_results) *n_results = static_cast<uint32_t>(cands.size());
  if (results)
    for (uint32_t i = 0; i < std::min<uint32_t>(cap, static_cast<uint32_t>(cands.size())); ++i) results[i] = cands[i];
  const ckmpm_status at = apply_tuning(s, *pick);
  if (at != CKMPM_OK) return at;
  // Applying the pick dropped the graphs of the last probed shape: capture the
  // chosen shape's chunk graph now (capture runs nothing), so that the first
  // ckmpm_step_async after tuning does not pay for it.
  CK_CUDA(s, build_graph(s, static_cast<int>(s->tune.graph_chunk), 0, &s->graph_chunk));
  return CKMPM_OK;
}

ckmpm_status ckmpm_get_counters(ckmpm_scene* s, uint64_t* out5) {
  if (!s || !out5) return fail(s, CKMPM_ERR_INVALID, "null argument");
  Scalars h{};
  CK_CUDA(s, cudaMemcpyAsync(&h, s->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  out5[0] = static_cast<uint64_t>(h.step);
  out5[1] = h.lost;
  out5[2] = h.window_skips;
  out5[3] = h.status;
  out5[4] = h.timeouts;
  return CKMPM_OK;
}

ckmpm_status ckmpm_get_time(ckmpm_scene* s, double* out2) {
  if (!s || !out2) return fail(s, CKMPM_ERR_INVALID, "null argument");
  Scalars h{};
  CK_CUDA(s, cudaMemcpyAsync(&h, s->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  out2[0] = h.time;
  out2[1] = h.frame_end;
  return CKMPM_OK;
}

// The grid the next substep reads and its epoch (the substep count).
static void dd_grid(ckmpm_scene* s, long long** g, int32_t** stamp, int32_t* epoch) {
  const int parity = static_cast<int>(s->host_step & 1);
  *g = s->grid.grid[parity];
  *stamp = s->grid.stamp[parity];
  *epoch = static_cast<int32_t>(s->host_step);
}

static ckmpm_status dd_check(ckmpm_scene* s) {
  if (!s) return fail(s, CKMPM_ERR_INVALID, "null scene");
  if (!s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (s->nstack != 1) return fail(s, CKMPM_ERR_INVALID, "a batch is not decomposed");
  return CKMPM_OK;
}

ckmpm_status ckmpm_dd_blocks(ckmpm_scene* s, uint32_t* n_blocks) {
  if (!s || !n_blocks) return fail(s, CKMPM_ERR_INVALID, "null argument");
  *n_blocks = s->sc.nblocks_domain;
  return CKMPM_OK;
}

ckmpm_status ckmpm_dd_mark(ckmpm_scene* s, int32_t* mask) {
  ckmpm_status st = dd_check(s);
  if (st != CKMPM_OK) return st;
  if (!mask) return fail(s, CKMPM_ERR_INVALID, "null argument");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  long long* g;
  int32_t* stamp;
  int32_t epoch;
  dd_grid(s, &g, &stamp, &epoch);
  dd_mark_kernel<<<s->sm_count * 4, 256, 0, s->stream>>>(stamp, epoch, s->sc.nblocks_domain, mask);
  CK_CUDA(s, cudaGetLastError());
  return CKMPM_OK;
}

ckmpm_status ckmpm_dd_pack(ckmpm_scene* s, const int32_t* blocks, uint32_t n, long long* buf) {
  ckmpm_status st = dd_check(s);
  if (st != CKMPM_OK) return st;
  if (n == 0) return CKMPM_OK;
  if (!blocks || !buf) return fail(s, CKMPM_ERR_INVALID, "null argument");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  long long* g;
  int32_t* stamp;
  int32_t epoch;
  dd_grid(s, &g, &stamp, &epoch);
  dd_pack_kernel<<<s->sm_count * 4, 256, 0, s->stream>>>(g, stamp, epoch, blocks, n, s->sc.nblocks_domain,
                                                         reinterpret_cast<longlong2*>(buf));
  CK_CUDA(s, cudaGetLastError());
  return CKMPM_OK;
}

ckmpm_status ckmpm_dd_unpack(ckmpm_scene* s, const int32_t* blocks, uint32_t n, const long long* buf) {
  ckmpm_status st = dd_check(s);
  if (st != CKMPM_OK) return st;
  if (n == 0) return CKMPM_OK;
  if (!blocks || !buf) return fail(s, CKMPM_ERR_INVALID, "null argument");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  long long* g;
  int32_t* stamp;
  int32_t epoch;
  dd_grid(s, &g, &stamp, &epoch);
  dd_unpack_kernel<<<s->sm_count * 4, 256, 0, s->stream>>>(g, stamp, epoch, blocks, n, s->sc.nblocks_domain,
                                                           reinterpret_cast<const longlong2*>(buf));
  CK_CUDA(s, cudaGetLastError());
  return CKMPM_OK;
}

ckmpm_status ckmpm_get_dt(ckmpm_scene* s, float* out2) {
  if (!s || !out2) return fail(s, CKMPM_ERR_INVALID, "null argument");
  Scalars h{};
  CK_CUDA(s, cudaMemcpyAsync(&h, s->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  out2[0] = h.cur_dt;
  out2[1] = h.next_dt;
  return CKMPM_OK;
}

ckmpm_status ckmpm_step_profiled(ckmpm_scene* s, uint32_t nsteps, float dt, double* ms_out3) {
  if (!s || !s->setup_done) return fail(s, CKMPM_ERR_INVALID, "ckmpm_setup has not run");
  if (!ms_out3) return fail(s, CKMPM_ERR_INVALID, "null argument");
  CK_CUDA(s, cudaSetDevice(s->desc.device));
  const uint64_t step = s->host_step;
  set_next_dt_kernel<<<1, 32, 0, s->stream>>>(s->scal, dt);
  std::vector<cudaEvent_t> ev;
  const size_t nm = s->models.size();
  ev.resize(nsteps * nm * 3);
  for (auto& x : ev) CK_CUDA(s, cudaEventCreate(&x));
  for (uint32_t i = 0; i < nsteps; ++i) {
    const int parity = static_cast<int>((step + i) & 1);
    for (size_t mi = 0; mi < nm; ++mi) {
      auto& m = s->models[mi];
      cudaEvent_t* E = &ev[(i * nm + mi) * 3];
      CK_CUDA(s, cudaEventRecord(E[0], s->stream));
      CK_CUDA(s, launch_fused_any(s, m));
      CK_CUDA(s, cudaEventRecord(E[1], s->stream));
      CK_CUDA(s, launch_compact(s, m, m.dev.bl[parity ^ 1]));
      if (mi + 1 == nm) CK_CUDA(s, launch_zero(s, parity ^ 1, parity, 2));
      CK_CUDA(s, cudaEventRecord(E[2], s->stream));
    }
    end_substep_kernel<<<1, 32, 0, s->stream>>>(s->scal);
    ++s->host_step;
  }
  CK_CUDA(s, cudaStreamSynchronize(s->stream));
  double fused = 0, other = 0;
  for (uint32_t i = 0; i < nsteps * nm; ++i) {
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, ev[i * 3], ev[i * 3 + 1]);
    cudaEventElapsedTime(&b, ev[i * 3 + 1], ev[i * 3 + 2]);
    fused += a;
    other += b;
  }
  for (auto& x : ev) cudaEventDestroy(x);
  ms_out3[0] = fused;
  ms_out3[1] = other;
  ms_out3[2] = static_cast<double>(nsteps * nm);
  return ckmpm_status_check(s);
}

ckmpm_status ckmpm_debug_constitutive(const ckmpm_material* material, uint32_t n, const float* C, float dt, float* F,
                                      float* aux, float* tau, float* U, float* S, float* V) {
  if (!material || !C || !F || !tau || n == 0) return fail(nullptr, CKMPM_ERR_INVALID, "null argument");
  MaterialParams mp{};
  mp.kind = material->kind;
  std::string why;
  if (!valid_material(*material, &why)) return fail(nullptr, CKMPM_ERR_INVALID, why);
  if (material->kind == CKMPM_LINEAR) return fail(nullptr, CKMPM_ERR_INVALID, "the linear model keeps a stored stress");
  for (int k = 0; k < kMaterialParams; ++k) mp.p[k] = material->p[k];
  float *dC, *dF, *dA, *dT, *dU, *dS, *dV;
  auto chk = [](cudaError_t e) { return e == cudaSuccess; };
  if (!chk(cudaMalloc(&dC, sizeof(float) * 9 * n)) || !chk(cudaMalloc(&dF, sizeof(float) * 9 * n)) ||
      !chk(cudaMalloc(&dA, sizeof(float) * n)) || !chk(cudaMalloc(&dT, sizeof(float) * 9 * n)) ||
      !chk(cudaMalloc(&dU, sizeof(float) * 9 * n)) || !chk(cudaMalloc(&dS, sizeof(float) * 3 * n)) ||
      !chk(cudaMalloc(&dV, sizeof(float) * 9 * n)))
    return fail(nullptr, CKMPM_ERR_CUDA, "allocation failed");
  cudaMemcpy(dC, C, sizeof(float) * 9 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dF, F, sizeof(float) * 9 * n, cudaMemcpyHostToDevice);
  if (aux) cudaMemcpy(dA, aux, sizeof(float) * n, cudaMemcpyHostToDevice);
  else cudaMemset(dA, 0, sizeof(float) * n);
  debug_constitutive_kernel<<<(n + 127) / 128, 128>>>(mp, n, dC, dt, dF, dA, dT, dU, dS, dV);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) {
    cudaMemcpy(F, dF, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost);
    if (aux) cudaMemcpy(aux, dA, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(tau, dT, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost);
    if (U) cudaMemcpy(U, dU, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost);
    if (S) cudaMemcpy(S, dS, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost);
    if (V) cudaMemcpy(V, dV, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost);
  }
  cudaFree(dC);
  cudaFree(dF);
  cudaFree(dA);
  cudaFree(dT);
  cudaFree(dU);
  cudaFree(dS);
  cudaFree(dV);
  if (e != cudaSuccess) return fail(nullptr, CKMPM_ERR_CUDA, cudaGetErrorString(e));
  return CKMPM_OK;
}

ckmpm_status ckmpm_destroy(ckmpm_scene* s) {
  if (!s) return CKMPM_OK;
  cudaSetDevice(s->desc.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->copy_stream) {
    cudaStreamSynchronize(s->copy_stream);
    cudaStreamDestroy(s->copy_stream);
    cudaEventDestroy(s->ev_probe);
    cudaEventDestroy(s->ev_copy);
  }
  if (s->export_count) release_pinned_word(s->export_count);
  for (auto& m : s->models) {
    if (m.io) cudaFree(m.io);
    if (m.ev_copied) cudaEventDestroy(m.ev_copied);
  }
  free_graphs(s);
  for (auto& p : s->allocs) cudaFree(p.first);
  if (s->own_stream) cudaStreamDestroy(s->own_stream);
  delete s;
  return CKMPM_OK;
}

}  // extern "C"
