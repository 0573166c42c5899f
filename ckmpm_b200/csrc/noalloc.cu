// ckmpm_simulate_noalloc: the one entry point of this library that allocates
// no memory at all.
//
// Some callers cannot call cudaMalloc: plugins hosted by runtimes that own the
// whole device memory budget through their own pool (an allocation behind the
// pool's back can fail or push the host over its limit), and loops that
// cannot afford the device-wide synchronisation a cudaMalloc / cudaFree may
// cause.  For them this entry point runs a complete small simulation -- setup
// and nsteps substeps of one model -- with every piece of scratch memory
// (grid, block tables, index lists, setup ordering buffers, work counters, flags) taken
// from one file-scope __device__ array of fixed size.  The caller passes its
// inputs and outputs as device pointers.  The same kernels as the allocating
// path run in the same order, so the outputs match ckmpm_create /
// ckmpm_add_model / ckmpm_setup / ckmpm_step / ckmpm_get_state on the same
// inputs.
//
// The call waits for its own work: it reads the binned and live particle
// counts back to the host and synchronises the caller's stream three times.
// So it cannot be recorded into a CUDA graph: on a stream that is capturing it
// returns CKMPM_ERR_INVALID before enqueuing anything, and the capture stays
// valid.
//
// Limits: one model of at most kNoAllocMaxParticles particles in a domain of
// at most kNoAllocMaxDomainBlocks 4^3-cell blocks; the array takes
// kNoAllocScratchBytes of device memory on every GPU that loads this library,
// until the process exits.  All calls share the array: calls that overlap on
// the GPU (different streams or threads) race and corrupt each other.
// This file is compiled in the same translation unit as engine.cu (see
// library.cu) and reuses its kernels and launch helpers.

namespace {

constexpr uint32_t kNoAllocMaxParticles = 65536;
constexpr uint32_t kNoAllocMaxDomainBlocks = 4096;
constexpr int kNoAllocMaxDevices = 64;

constexpr size_t na_align(size_t b) { return (b + 255) & ~size_t(255); }

// Bytes of every region at the maximum sizes (see carve() below).
constexpr size_t kNaGrid = na_align(sizeof(long long) * 512 * kNoAllocMaxDomainBlocks);
constexpr size_t kNaDomainU32 = na_align(sizeof(uint32_t) * kNoAllocMaxDomainBlocks);
constexpr size_t kNaParticleU32 = na_align(sizeof(uint32_t) * kNoAllocMaxParticles);
constexpr size_t kNaParticleU16 = na_align(sizeof(uint16_t) * kNoAllocMaxParticles);
constexpr size_t kNaSlots = kNoAllocMaxDomainBlocks;  // slots <= min(domain blocks, particles)
constexpr size_t kNaBlockList = na_align(sizeof(int4) * kNaSlots) + 2 * na_align(sizeof(uint32_t) * kNaSlots) +
                                kNaDomainU32 + na_align(sizeof(uint32_t) * 28 * kNaSlots) + kNaParticleU16 +
                                2 * na_align(sizeof(uint32_t));
constexpr size_t kNaState = 14 * kNaParticleU32;  // x[3], F[9], aux, id
constexpr size_t kNoAllocScratchBytes =
    2 * kNaGrid + 2 * kNaDomainU32 + na_align(sizeof(Scalars)) + 2 * kNaState + 2 * kNaBlockList +
    kNaDomainU32 /*dense totals*/ + na_align(sizeof(uint32_t) * 2 * 64) /*tile sums*/ + na_align(4) /*ticket*/ +
    3 * kNaParticleU32 /*initial velocities*/ +
    3 * kNaParticleU32 /*setup: flat block indices, placement cursors, particle order*/ +
    18 * kNaParticleU32 /*export*/;

static_assert(kNoAllocScratchBytes < (size_t(56) << 20), "no-alloc scratch must stay modest");

// The scratch.  In host code `g_noalloc_scratch` is only a host-side stand-in
// for the symbol, not a device address: its device address comes from
// cudaGetSymbolAddress, per device, in na_base().
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

unsigned char* g_na_base[kNoAllocMaxDevices] = {};
int g_na_ctas[kNoAllocMaxDevices] = {};
std::mutex g_na_mutex;  // host threads making a first call at the same time

// Per-device set-up, done by the first call on each device with that device
// current: the device address of the scratch array and the persistent grid size.
cudaError_t na_base(int device, unsigned char** base, int* ctas) {
  if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_base[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    const void* fns[5] = {reinterpret_cast<const void*>(g2p2g_kernel<kFixedCorotated, kFusedThreads>),
                          reinterpret_cast<const void*>(g2p2g_kernel<kDruckerPrager, kFusedThreads>),
                          reinterpret_cast<const void*>(g2p2g_kernel<kFluid, kFusedThreads>),
                          reinterpret_cast<const void*>(g2p2g_kernel<kVonMises, kFusedThreads>),
                          reinterpret_cast<const void*>(g2p2g_kernel<kNacc, kFusedThreads>)};
    int lowest = 1 << 30;
    for (const void* fn : fns) {
      int occ = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kFusedThreads, kSmemFused);
      lowest = std::min(lowest, occ);
    }
    g_na_ctas[device] = std::max(1, lowest) * sms;
    g_na_base[device] = static_cast<unsigned char*>(p);
  }
  *base = g_na_base[device];
  *ctas = g_na_ctas[device];
  return cudaSuccess;
}

struct NaCarver {
  unsigned char* p;
  template <typename T>
  T* take(size_t count) {
    T* r = reinterpret_cast<T*>(p);
    p += na_align(sizeof(T) * count);
    return r;
  }
};

// Scatter the block-ordered export back to input order.
__global__ void noalloc_scatter_kernel(uint32_t n, const uint32_t* __restrict__ id, const float* __restrict__ bx,
                                       const float* __restrict__ bv, const float* __restrict__ bF,
                                       const float* __restrict__ ba, float* x, float* v, float* F, float* aux,
                                       uint32_t n_in, int has_F, int has_aux) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t d = id[i];
  if (d >= n_in) return;
  if (x)
    for (int k = 0; k < 3; ++k) x[3 * d + k] = bx[3 * i + k];
  if (v)
    for (int k = 0; k < 3; ++k) v[3 * d + k] = bv[3 * i + k];
  if (F)
    for (int k = 0; k < 9; ++k) F[9 * d + k] = has_F ? bF[9 * i + k] : ((k & 3) ? 0.f : 1.f);
  if (aux) aux[d] = has_aux ? ba[i] : 0.f;
}

// Marks every output slot as not written (NaN) before the scatter, so that
// particles lost to the domain edge stay recognisable.
__global__ void noalloc_fill_kernel(uint32_t n, float* x, float* v, float* F, float* aux) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float nan = __int_as_float(0x7fc00000);
  if (x)
    for (int k = 0; k < 3; ++k) x[3 * i + k] = nan;
  if (v)
    for (int k = 0; k < 3; ++k) v[3 * i + k] = nan;
  if (F)
    for (int k = 0; k < 9; ++k) F[9 * i + k] = nan;
  if (aux) aux[i] = nan;
}

ckmpm_status na_fail(const char** message, ckmpm_status code, const char* text) {
  if (message) *message = text;
  return code;
}

}  // namespace

extern "C" ckmpm_status ckmpm_simulate_noalloc(const ckmpm_scene_desc* desc, const ckmpm_material* material,
                                               uint32_t n, const float* x, const float* v, uint32_t nv, float mass,
                                               float volume, uint32_t nsteps, float dt, void* cuda_stream,
                                               float* x_out, float* v_out, float* F_out, float* aux_out,
                                               uint32_t* n_live, const char** message) {
  if (message) *message = "ok";
  if (!desc || !material || !x || !v) return na_fail(message, CKMPM_ERR_INVALID, "null argument");
  if (n == 0) return na_fail(message, CKMPM_ERR_INVALID, "empty model");
  if (n > kNoAllocMaxParticles)
    return na_fail(message, CKMPM_ERR_CAPACITY, "more particles than the no-alloc limit (65536)");
  if (nv != 1 && nv != n) return na_fail(message, CKMPM_ERR_INVALID, "nv must be 1 or n");
  if (!(desc->dx > 0.f)) return na_fail(message, CKMPM_ERR_INVALID, "dx must be positive");
  for (int a = 0; a < 3; ++a)
    if (desc->domain_blocks[a] < 1) return na_fail(message, CKMPM_ERR_INVALID, "domain_blocks out of range");
  const uint64_t nbd64 =
      static_cast<uint64_t>(desc->domain_blocks[0]) * desc->domain_blocks[1] * desc->domain_blocks[2];
  if (nbd64 > kNoAllocMaxDomainBlocks)
    return na_fail(message, CKMPM_ERR_CAPACITY, "domain larger than the no-alloc limit (4096 blocks)");
  if (desc->boundary != CKMPM_BOUNDARY_STICKY_BLOCKS && desc->boundary != CKMPM_BOUNDARY_SLIP_FLOOR)
    return na_fail(message, CKMPM_ERR_INVALID, "unknown boundary kind");
  if (desc->max_particles_per_block > static_cast<uint32_t>(kMaxParticlesPerBlock))
    return na_fail(message, CKMPM_ERR_INVALID, "max_particles_per_block > 4096");
  if (material->kind != CKMPM_FIXED_COROTATED && material->kind != CKMPM_DRUCKER_PRAGER &&
      material->kind != CKMPM_FLUID && material->kind != CKMPM_VON_MISES && material->kind != CKMPM_NACC)
    return na_fail(message, CKMPM_ERR_INVALID, "unsupported material kind (the linear model keeps a stored stress)");
  if (!(mass > 0.f) || !(volume > 0.f)) return na_fail(message, CKMPM_ERR_INVALID, "mass and volume must be positive");
  if (!(dt >= 0.f)) return na_fail(message, CKMPM_ERR_INVALID, "dt must be non-negative");

  int prev_device = 0;
  if (cudaGetDevice(&prev_device) != cudaSuccess) return na_fail(message, CKMPM_ERR_CUDA, "cudaGetDevice failed");
  if (cudaSetDevice(desc->device) != cudaSuccess) return na_fail(message, CKMPM_ERR_CUDA, "cudaSetDevice failed");
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev_device};
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  // The call synchronises its stream and reads counts back to the host, which a
  // stream capture cannot record: refuse before enqueuing anything.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &capture) != cudaSuccess)
    return na_fail(message, CKMPM_ERR_CUDA, "cudaStreamIsCapturing failed");
  if (capture != cudaStreamCaptureStatusNone)
    return na_fail(message, CKMPM_ERR_INVALID,
                   "the stream is capturing a CUDA graph; this call synchronises its stream and cannot be captured");
  unsigned char* base = nullptr;
  int ctas = 0;
  if (na_base(desc->device, &base, &ctas) != cudaSuccess)
    return na_fail(message, CKMPM_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
  const uint32_t nbd = static_cast<uint32_t>(nbd64);

  // Scene constants, as ckmpm_create computes them.
  SceneDev sc{};
  sc.dx = desc->dx;
  sc.inv_dx = static_cast<float>(1.0 / static_cast<double>(desc->dx));
  for (int a = 0; a < 3; ++a) sc.dims[a] = desc->domain_blocks[a];
  sc.gravity = desc->gravity;
  sc.mass_clamp = desc->mass_clamp;
  sc.boundary = desc->boundary;
  sc.floor_cells = desc->floor_cells;
  sc.grid_unit = mass * kFixInvScale;
  init_colour_classes(sc, 1);

  // Carve the scratch array (fixed layout at the maximum sizes).
  NaCarver cv{base};
  GridDev grid{};
  Scalars* scal = nullptr;
  ModelDev d{};
  const bool hasF = material->kind != CKMPM_FLUID;
  const bool hasAux = material->kind != CKMPM_FIXED_COROTATED;
  for (int b = 0; b < 2; ++b) grid.grid[b] = cv.take<long long>(size_t(512) * kNoAllocMaxDomainBlocks);
  for (int b = 0; b < 2; ++b) grid.stamp[b] = cv.take<int32_t>(kNoAllocMaxDomainBlocks);
  scal = cv.take<Scalars>(1);
  for (int b = 0; b < 2; ++b) {
    StateDev& s = d.st[b];
    for (int a = 0; a < 3; ++a) s.x[a] = cv.take<float>(kNoAllocMaxParticles);
    for (int k = 0; k < 9; ++k) {
      float* f = cv.take<float>(kNoAllocMaxParticles);
      s.F[k] = hasF ? f : nullptr;
    }
    float* a = cv.take<float>(kNoAllocMaxParticles);
    s.aux = hasAux ? a : nullptr;
    s.id = cv.take<uint32_t>(kNoAllocMaxParticles);
  }
  for (int b = 0; b < 2; ++b) {
    BlockListDev& bl = d.bl[b];
    bl.keys = cv.take<int4>(kNaSlots);
    bl.start = cv.take<uint32_t>(kNaSlots);
    bl.count = cv.take<uint32_t>(kNaSlots);
    bl.table = cv.take<int32_t>(kNoAllocMaxDomainBlocks);
    bl.prefix28 = cv.take<uint32_t>(28 * kNaSlots);
    bl.idx = cv.take<uint16_t>(kNoAllocMaxParticles);
    bl.nblocks = cv.take<uint32_t>(1);
    bl.nparticles = cv.take<uint32_t>(1);
  }
  d.dense_total = cv.take<uint32_t>(kNoAllocMaxDomainBlocks);
  d.tile_sums = cv.take<uint32_t>(2 * 64);
  d.ticket = cv.take<uint32_t>(1);
  d.vel_in = cv.take<float>(3 * size_t(kNoAllocMaxParticles));
  uint32_t* flat = cv.take<uint32_t>(kNoAllocMaxParticles);
  uint32_t* cursor = cv.take<uint32_t>(kNoAllocMaxParticles);
  uint32_t* perm = cv.take<uint32_t>(kNoAllocMaxParticles);
  float* ex = cv.take<float>(3 * size_t(kNoAllocMaxParticles));
  float* ev = cv.take<float>(3 * size_t(kNoAllocMaxParticles));
  float* eF = cv.take<float>(9 * size_t(kNoAllocMaxParticles));
  float* ea = cv.take<float>(kNoAllocMaxParticles);
  uint32_t* eid = cv.take<uint32_t>(kNoAllocMaxParticles);
  if (static_cast<size_t>(cv.p - base) > kNoAllocScratchBytes)
    return na_fail(message, CKMPM_ERR_CAPACITY, "no-alloc scratch layout overflow");

  d.cap_particles = n;
  d.cap_slots = std::max<uint32_t>(1, std::min<uint32_t>(nbd, n));
  d.max_per_block = desc->max_particles_per_block ? desc->max_particles_per_block : kMaxParticlesPerBlock;
  d.track_ids = 1;
  d.mat.kind = material->kind;
  for (int k = 0; k < kMaterialParams; ++k) d.mat.p[k] = material->p[k];
  d.mass = mass;
  d.vol = volume;
  d.flush_ratio = 1.0;
  const uint32_t ntiles = (nbd + kCompactTile - 1) / kCompactTile;

#define NA_CUDA(call)                                                   \
  do {                                                                  \
    if ((call) != cudaSuccess) return na_fail(message, CKMPM_ERR_CUDA, #call " failed"); \
  } while (0)

  // Clear what must start at zero (the array keeps the previous call's contents).
  for (int b = 0; b < 2; ++b) NA_CUDA(cudaMemsetAsync(grid.stamp[b], 0xFF, sizeof(int32_t) * nbd, st));
  NA_CUDA(cudaMemsetAsync(scal, 0, sizeof(Scalars), st));
  for (int b = 0; b < 2; ++b) {
    NA_CUDA(cudaMemsetAsync(d.bl[b].nblocks, 0, sizeof(uint32_t), st));
    NA_CUDA(cudaMemsetAsync(d.bl[b].nparticles, 0, sizeof(uint32_t), st));
  }
  NA_CUDA(cudaMemsetAsync(d.dense_total, 0, sizeof(uint32_t) * nbd, st));
  NA_CUDA(cudaMemsetAsync(d.ticket, 0, sizeof(uint32_t), st));

  // Setup: bin, compact, place and order each block's particles, gather,
  // identity previous step, initial grid -- the sequence of ckmpm_setup.
  setup_bin_kernel<<<(n + 255) / 256, 256, 0, st>>>(sc, n, x, nullptr, flat, d.dense_total);
  compact_reduce_kernel<<<ntiles, kCompactThreads, 0, st>>>(sc, d.dense_total, d.tile_sums);
  compact_scatter_kernel<<<ntiles, kCompactThreads, 0, st>>>(sc, d.dense_total, d.tile_sums, d.bl[0], d.cap_slots,
                                                             d.ticket, scal);
  NA_CUDA(cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * d.cap_slots, st));
  setup_place_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, flat, d.bl[0], cursor, perm);
  setup_order_kernel<256><<<ctas, 256, 0, st>>>(sc, d.bl[0], x, perm, scal);
  uint32_t counts[2] = {0, 0};
  NA_CUDA(cudaMemcpyAsync(&counts[0], d.bl[0].nblocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(&counts[1], d.bl[0].nparticles, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  const uint32_t n_valid = counts[1];
  const float aux0 = material->kind == CKMPM_FLUID ? material->p[3]
                     : material->kind == CKMPM_NACC ? material->p[2]
                     : material->kind == CKMPM_VON_MISES ? 1.f : 0.f;
  if (n_valid > 0)
    setup_gather_kernel<<<(n_valid + 255) / 256, 256, 0, st>>>(d, 1, n_valid, perm, x, v, nv, aux0, 0u);
  NA_CUDA(cudaMemcpyAsync(d.bl[1].table, d.bl[0].table, sizeof(int32_t) * nbd, cudaMemcpyDeviceToDevice, st));
  NA_CUDA(cudaMemcpyAsync(d.bl[1].start, d.bl[0].start, sizeof(uint32_t) * d.cap_slots, cudaMemcpyDeviceToDevice, st));
  NA_CUDA(cudaMemcpyAsync(d.bl[1].count, d.bl[0].count, sizeof(uint32_t) * d.cap_slots, cudaMemcpyDeviceToDevice, st));
  NA_CUDA(cudaMemcpyAsync(d.bl[1].keys, d.bl[0].keys, sizeof(int4) * d.cap_slots, cudaMemcpyDeviceToDevice, st));
  NA_CUDA(cudaMemcpyAsync(d.bl[1].nblocks, d.bl[0].nblocks, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  NA_CUDA(cudaMemcpyAsync(d.bl[1].nparticles, d.bl[0].nparticles, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  if (counts[0] > 0) setup_identity_kernel<<<counts[0], 256, 0, st>>>(d.bl[0], d.bl[1]);
  NA_CUDA(cudaMemsetAsync(d.ticket, 0, sizeof(uint32_t), st));
  int sms = 0;
  NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, desc->device));
  zero_windows_kernel<<<sms * 4, 256, 0, st>>>(sc, d.bl[0], grid.grid[0], grid.stamp[0], scal, 0);
  rasterize_kernel<kFusedThreads><<<ctas, kFusedThreads, kSmemFused, st>>>(sc, d, grid, scal);
  NA_CUDA(cudaMemsetAsync(d.ticket, 0, sizeof(uint32_t), st));
  zero_windows_kernel<<<sms * 4, 256, 0, st>>>(sc, d.bl[0], grid.grid[1], grid.stamp[1], scal, 1);
  finish_setup_kernel<<<1, 32, 0, st>>>(scal, n - n_valid, 0.f, 0.f, 0.f);  // keeps setup's status bits
  NA_CUDA(cudaGetLastError());

  // Substeps: the launch sequence of ckmpm_step without graphs.
  if (nsteps > 0) set_next_dt_kernel<<<1, 32, 0, st>>>(scal, dt);
  for (uint32_t i = 0; i < nsteps; ++i) {
    const int parity = static_cast<int>(i & 1);
    switch (material->kind) {
      case CKMPM_FIXED_COROTATED:
        g2p2g_kernel<kFixedCorotated, kFusedThreads><<<ctas, kFusedThreads, kSmemFused, st>>>(sc, d, grid, scal);
        break;
      case CKMPM_DRUCKER_PRAGER:
        g2p2g_kernel<kDruckerPrager, kFusedThreads><<<ctas, kFusedThreads, kSmemFused, st>>>(sc, d, grid, scal);
        break;
      case CKMPM_VON_MISES:
        g2p2g_kernel<kVonMises, kFusedThreads><<<ctas, kFusedThreads, kSmemFused, st>>>(sc, d, grid, scal);
        break;
      case CKMPM_NACC:
        g2p2g_kernel<kNacc, kFusedThreads><<<ctas, kFusedThreads, kSmemFused, st>>>(sc, d, grid, scal);
        break;
      default:
        g2p2g_kernel<kFluid, kFusedThreads><<<ctas, kFusedThreads, kSmemFused, st>>>(sc, d, grid, scal);
    }
    compact_reduce_kernel<<<ntiles, kCompactThreads, 0, st>>>(sc, d.dense_total, d.tile_sums);
    compact_scatter_kernel<<<ntiles, kCompactThreads, 0, st>>>(sc, d.dense_total, d.tile_sums, d.bl[parity ^ 1],
                                                               d.cap_slots, d.ticket, scal);
    zero_windows_kernel<<<sms * 4, 256, 0, st>>>(sc, d.bl[parity ^ 1], grid.grid[parity], grid.stamp[parity], scal, 2);
    end_substep_kernel<<<1, 32, 0, st>>>(scal);
  }
  NA_CUDA(cudaGetLastError());

  // Export: gather in block order, then scatter to the caller's arrays in input order.
  const BlockListDev& cur = d.bl[nsteps & 1];
  uint32_t live = 0;
  NA_CUDA(cudaMemcpyAsync(&live, cur.nparticles, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  probe_kernel<kProbeThreads><<<sms * 4, kProbeThreads, kSmemVTile, st>>>(sc, d, grid, scal, ex, ev, hasF ? eF : nullptr,
                                                                         hasAux ? ea : nullptr, eid, nullptr);
  NA_CUDA(cudaStreamSynchronize(st));
  if (x_out || v_out || F_out || aux_out) {
    noalloc_fill_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, x_out, v_out, F_out, aux_out);
    if (live > 0)
      noalloc_scatter_kernel<<<(live + 255) / 256, 256, 0, st>>>(live, eid, ex, ev, eF, ea, x_out, v_out, F_out,
                                                                 aux_out, n, hasF ? 1 : 0, hasAux ? 1 : 0);
  }
  Scalars r{};
  NA_CUDA(cudaMemcpyAsync(&r, scal, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  NA_CUDA(cudaGetLastError());
#undef NA_CUDA
  if (n_live) *n_live = live;
  if (r.status & kStatusTimeout) return na_fail(message, CKMPM_ERR_TIMEOUT, "a bounded device wait gave up");
  if (r.status & kStatusCapacity) return na_fail(message, CKMPM_ERR_CAPACITY, "block capacity exceeded");
  if (r.status & kStatusNumeric) return na_fail(message, CKMPM_ERR_NUMERIC, "non-finite or out-of-range values");
  if (r.status & kStatusConsistency) return na_fail(message, CKMPM_ERR_INVALID, "rebin consistency check failed");
  if (r.status & kStatusOutsideBlock)
    return na_fail(message, CKMPM_ERR_NUMERIC, "a particle was outside the stencil window of its block");
  return CKMPM_OK;
}
