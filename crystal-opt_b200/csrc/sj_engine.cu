// sj_engine.cu -- host orchestration behind the C ABI (include/starjoin.h).
//
// Mirrors the reference's runQuery (src/ssb-jo/q33/0-lip.cu:205-302): reserve the
// dimension tables and filters, zero them, build, probe, read back the groups.
// Differences by design: integer status codes instead of CubDebugExit aborts,
// stream-ordered allocation from an engine-owned memory pool (no per-query
// cudaMalloc, no leaks), one zeroing memset per query instead of six, all
// filter/group geometry decided on the device, and compact group rows instead of
// the 437,500-slot dense result array.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "sj_datagen.h"
#include "sj_internal.h"

namespace sj {
uint32_t probe_smem_bytes(const SjProbeGeom& g);
cudaError_t launch_probe(const SjPlanRt& P, const SjProbeGeom& G, uint32_t rows_per_thread, cudaStream_t st,
                         const L2Window& w, bool pdl);
cudaError_t launch_finalize(const SjPlanRt& P, uint32_t group_capacity, cudaStream_t st, bool pdl);
__global__ void sj_dim_scan(const __grid_constant__ SjPlanRt P);
__global__ void sj_clear_head(uint4* __restrict__ head, uint64_t n16);
__global__ void sj_dim_insert(const __grid_constant__ SjPlanRt P);
}  // namespace sj

using namespace sj;

// ---------------------------------------------------------------- errors ----
static thread_local std::string g_last_error;

static sj_status fail(sj_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

#define SJ_CUDA(call)                                                                             \
  do {                                                                                            \
    cudaError_t _e = (call);                                                                      \
    if (_e != cudaSuccess) {                                                                      \
      if (_e == cudaErrorMemoryAllocation) {                                                      \
        cudaGetLastError();                                                                       \
        return fail(SJ_ERR_OUT_OF_MEMORY, "%s: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, \
                    __LINE__);                                                                    \
      }                                                                                           \
      return fail(SJ_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
    }                                                                                             \
  } while (0)

extern "C" const char* sj_status_string(sj_status s) {
  switch (s) {
    case SJ_OK: return "ok";
    case SJ_ERR_INVALID_ARGUMENT: return "invalid argument";
    case SJ_ERR_UNSUPPORTED: return "unsupported";
    case SJ_ERR_OUT_OF_MEMORY: return "out of device memory";
    case SJ_ERR_CUDA: return "CUDA error";
    case SJ_ERR_CAPACITY: return "result buffer too small";
    case SJ_ERR_TIMEOUT: return "device wait timed out";
    case SJ_ERR_NO_DEVICE: return "no CUDA device";
    case SJ_ERR_REJECTED: return "rejected by admission control";
    case SJ_ERR_CANCELLED: return "cancelled";
  }
  return "unknown status";
}

extern "C" const char* sj_last_error(void) { return g_last_error.c_str(); }

namespace sj {
sj_status set_error(sj_status s, const char* msg) {
  g_last_error = msg;
  return s;
}
}  // namespace sj

// ---------------------------------------------------------------- engine ----

// Persisting-L2 set-aside for the probes' access-policy windows, shared by every
// engine of this process on a device: the first engine reserves it (at most
// kL2PersistWant, within the device maximum) and the last one gives the
// previous limit back.  The limit belongs to this process's CUDA context; where
// it cannot be changed (MPS, MIG) the probes launch without windows.
namespace {
#ifndef SJ_L2_PERSIST_MB
#define SJ_L2_PERSIST_MB 48
#endif
constexpr size_t kL2PersistWant = (size_t)SJ_L2_PERSIST_MB << 20;
std::mutex g_l2_mu;
struct L2Reservation {
  int users = 0;
  size_t prev = 0, held = 0;
};
L2Reservation g_l2[64];

size_t l2_acquire(int device) {
  std::lock_guard<std::mutex> g(g_l2_mu);
  L2Reservation& r = g_l2[device & 63];
  if (r.users++ == 0) {
    int max_persist = 0;
    r.held = 0;
    if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, device) == cudaSuccess &&
        max_persist > 0 && cudaDeviceGetLimit(&r.prev, cudaLimitPersistingL2CacheSize) == cudaSuccess) {
      const size_t want = std::min<size_t>(kL2PersistWant, (size_t)max_persist);
      if (want > r.prev && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess) r.held = want;
      else if (r.prev > 0) r.held = r.prev;  // an existing set-aside is used as it is
    }
    cudaGetLastError();
  }
  return r.held;
}

void l2_release(int device) {
  std::lock_guard<std::mutex> g(g_l2_mu);
  L2Reservation& r = g_l2[device & 63];
  if (r.users > 0 && --r.users == 0) {
    if (r.held && r.held != r.prev) {
      cudaCtxResetPersistingL2Cache();
      cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, r.prev);
    }
    r.held = 0;
    cudaGetLastError();
  }
}
}  // namespace

extern "C" sj_status sj_engine_create(int device, sj_engine** out) {
  if (!out) return fail(SJ_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(SJ_ERR_NO_DEVICE, "no CUDA device visible (%s)", cudaGetErrorString(e));
  }
  if (device < 0 || device >= n) return fail(SJ_ERR_INVALID_ARGUMENT, "device %d out of range", device);
  SJ_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  SJ_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(SJ_ERR_UNSUPPORTED, "device %d is sm_%d%d; this build targets sm_100a", device,
                                   prop.major, prop.minor);
  sj_engine* eng = new sj_engine();
  eng->device = device;
  eng->sm_count = prop.multiProcessorCount;
  eng->smem_optin = prop.sharedMemPerBlockOptin;
  eng->l2_window_max = prop.accessPolicyMaxWindowSize > 0 ? (size_t)prop.accessPolicyMaxWindowSize : 0;
  cudaMemPoolProps pp;
  memset(&pp, 0, sizeof(pp));
  pp.allocType = cudaMemAllocationTypePinned;
  pp.handleTypes = cudaMemHandleTypeNone;
  pp.location.type = cudaMemLocationTypeDevice;
  pp.location.id = device;
  e = cudaMemPoolCreate(&eng->pool, &pp);
  if (e != cudaSuccess) {
    delete eng;
    return fail(SJ_ERR_CUDA, "cudaMemPoolCreate: %s", cudaGetErrorString(e));
  }
  uint64_t thr = ~0ull;  // keep freed blocks for reuse by later queries
  cudaMemPoolSetAttribute(eng->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  e = cudaStreamCreateWithFlags(&eng->copy_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaMemPoolDestroy(eng->pool);
    delete eng;
    return fail(SJ_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  eng->l2_persist_bytes = l2_acquire(device);
  *out = eng;
  return SJ_OK;
}

extern "C" void sj_engine_destroy(sj_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  cudaDeviceSynchronize();
  if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
  if (e->pool) cudaMemPoolDestroy(e->pool);
  l2_release(e->device);
  delete e;
}

extern "C" int sj_device_sm_count(sj_engine* e) { return e ? e->sm_count : 0; }

// ----------------------------------------------------------------- query ----
struct sj_query {
  sj_engine* eng = nullptr;
  sj_plan plan;
  SjPlanRt rt;
  SjProbeGeom geom;
  uint32_t rows_per_thread = 4;
  uint8_t* arena = nullptr;
  size_t arena_bytes = 0;
  size_t zero_bytes = 0;     // the whole zeroed region (first build, after an error)
  size_t head_bytes = 0;     // descriptor and payload bitmaps: cleared by every build
  bool groups_clean = false; // the group sums are zero (the compaction kernel leaves them so)
  uint64_t group_capacity = 0;
  std::vector<uint32_t> in_bitmaps;  // host staging, SJ_MAX_DIMS x 128 words
  cudaEvent_t ev_start = nullptr, ev_built = nullptr, ev_probed = nullptr;
  bool built = false, probed = false;
  bool probed_since_build = false;  // a further probe clears the probe's counters and the result count first
  cudaStream_t stream = nullptr;
  L2Window l2win;  // the probe's window over the hash tables and filters
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

static sj_status validate_plan(const sj_plan* p) {
  if (!p) return fail(SJ_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (p->n_dims < 1 || p->n_dims > SJ_MAX_DIMS) return fail(SJ_ERR_INVALID_ARGUMENT, "n_dims=%d", p->n_dims);
  if (!p->measure) return fail(SJ_ERR_INVALID_ARGUMENT, "measure column is NULL");
  if (p->fact_rows < 0 || p->fact_rows > 0xFFFFFFF0ll)
    return fail(SJ_ERR_UNSUPPORTED, "fact_rows=%lld (max 2^32-16)", (long long)p->fact_rows);
  const int64_t end = p->row_end < 0 ? p->fact_rows : p->row_end;
  if (p->row_begin < 0 || end < p->row_begin || end > p->fact_rows)
    return fail(SJ_ERR_INVALID_ARGUMENT, "row range [%lld, %lld) outside [0, %lld)", (long long)p->row_begin,
                (long long)end, (long long)p->fact_rows);
  int used[SJ_MAX_DIMS] = {0};
  for (int i = 0; i < p->n_dims; ++i) {
    const int d = p->order[i];
    if (d < 0 || d >= p->n_dims || used[d]) return fail(SJ_ERR_INVALID_ARGUMENT, "order is not a permutation");
    used[d] = 1;
  }
  if (p->bf_bits_per_key < SJ_BF_AUTO || p->bf_bits_per_key > 64)
    return fail(SJ_ERR_INVALID_ARGUMENT, "bf_bits_per_key=%d", p->bf_bits_per_key);
  if (p->bf_bits_per_key != 0 && (p->bf_hashes < 1 || p->bf_hashes > 4))
    return fail(SJ_ERR_INVALID_ARGUMENT, "bf_hashes=%d (1..4)", p->bf_hashes);
  uint64_t groups = 1;
  for (int d = 0; d < p->n_dims; ++d) {
    const sj_dim& D = p->dims[d];
    if (!D.fact_fk || !D.key) return fail(SJ_ERR_INVALID_ARGUMENT, "dim %d: NULL column", d);
    if (!aligned16(D.fact_fk)) return fail(SJ_ERR_INVALID_ARGUMENT, "dim %d: fact column not 16-byte aligned", d);
    if (D.rows < 0 || D.rows > 0x7FFFFFFFll) return fail(SJ_ERR_INVALID_ARGUMENT, "dim %d: rows", d);
    if (D.ht_len <= 0) return fail(SJ_ERR_INVALID_ARGUMENT, "dim %d: ht_len=%d", d, D.ht_len);
    if (D.pred_kind < SJ_PRED_ALL || D.pred_kind > SJ_PRED_RANGE)
      return fail(SJ_ERR_INVALID_ARGUMENT, "dim %d: pred_kind", d);
    if (D.pred_kind != SJ_PRED_ALL && !D.filter_attr)
      return fail(SJ_ERR_INVALID_ARGUMENT, "dim %d: predicate without filter_attr", d);
    if (D.pred_kind == SJ_PRED_IN) {
      if (D.in_count < 0 || (D.in_count > 0 && !D.in_codes)) return fail(SJ_ERR_INVALID_ARGUMENT, "dim %d: IN", d);
      for (int i = 0; i < D.in_count; ++i)
        if (D.in_codes[i] < 0 || D.in_codes[i] >= SJ_MAX_IN_CODES)
          return fail(SJ_ERR_UNSUPPORTED, "dim %d: IN code %d outside [0, %d)", d, D.in_codes[i], SJ_MAX_IN_CODES);
    }
    if (D.group) {
      if (!D.payload) return fail(SJ_ERR_INVALID_ARGUMENT, "dim %d: grouped without payload", d);
      const int64_t span = (int64_t)D.payload_max - D.payload_min + 1;
      if (span < 1 || span > SJ_MAX_PAYLOAD_SPAN)
        return fail(SJ_ERR_UNSUPPORTED, "dim %d: payload span %lld (1..%d)", d, (long long)span, SJ_MAX_PAYLOAD_SPAN);
      groups *= (uint64_t)span;
      if (groups > (1ull << 26)) return fail(SJ_ERR_UNSUPPORTED, "group space exceeds 2^26");
    }
  }
  if (!aligned16(p->measure)) return fail(SJ_ERR_INVALID_ARGUMENT, "measure column not 16-byte aligned");
  return SJ_OK;
}

// Shrink the ring depth, the chunk, then the filter budget, until the layout fits the
// shared memory of ctas_per_sm CTAs (1 KB per CTA is reserved by the runtime).
static void fit_geom(sj_engine* eng, SjProbeGeom& g, uint32_t ctas_per_sm, uint32_t pass) {
  const size_t limit = std::min<size_t>(eng->smem_optin, 233472 / std::max<uint32_t>(1, ctas_per_sm) - 1024);
  g.smem_bytes = probe_smem_bytes(g);
  while (g.smem_bytes > limit) {
    if (g.stages > 2) --g.stages;
    else if (g.chunk_rows > pass) g.chunk_rows -= pass;
    else if (g.bf_smem_bytes >= 4096) g.bf_smem_bytes /= 2;
    else if (g.bf_smem_bytes) g.bf_smem_bytes = 0;
    else if (g.group_smem_cap > 64) g.group_smem_cap /= 2;
    else break;
    g.smem_bytes = probe_smem_bytes(g);
  }
}

// Probe launch geometry.  tune.threads is the CTA size (256, 512 or 768): one
// producer warp plus 7, 15 or 23 consumer warps (a multiple of four warps, so the
// register file splits evenly over the SM's four sub-partitions).  A pass covers
// 32 * rows_per_lane rows per consumer warp; a chunk is a whole number of passes
// of every consumer warp.
static void default_geom(sj_engine* eng, const sj_plan* p, SjProbeGeom& g, uint32_t& rpl) {
  const sj_tuning& t = p->tune;
  const uint32_t threads = t.threads ? (uint32_t)t.threads : 512u;
  const uint32_t nwc = threads / 32 - 1;
  g.threads = (nwc + 1) * 32;
  rpl = (t.compact_threshold == 16 && nwc <= 15) ? 16u : 8u;
  const uint32_t pass = nwc * 32 * rpl;
  g.chunk_rows = t.chunk_rows ? (uint32_t)t.chunk_rows : 4 * pass;
  if (g.chunk_rows % pass) g.chunk_rows = (g.chunk_rows / pass + 1) * pass;
  g.stages = t.stages ? (uint32_t)t.stages : 2u;
  g.bf_smem_bytes = t.bf_smem_bytes ? (uint32_t)t.bf_smem_bytes : 40u * 1024u;
  g.group_smem_cap = 1024;
  uint32_t q1 = 1;
  while (q1 < 2 * 32 * rpl) q1 <<= 1;
  g.q1_cap = q1;
  g.q2_cap = 128;  // room for a two-survivors-per-lane Q1 round (64) over a partial Q2
  g.reorder_period = 16;
  const uint32_t per_sm = t.ctas_per_sm ? (uint32_t)t.ctas_per_sm : 1u;
  g.grid = (uint32_t)eng->sm_count * per_sm;
  fit_geom(eng, g, per_sm, pass);
}

static sj_status check_geom(sj_engine* eng, SjProbeGeom& g, uint32_t rpl) {
  const uint32_t nwc = g.threads / 32 - 1;
  const bool ok = ((nwc == 7 || nwc == 15) && (rpl == 8 || rpl == 16)) || (nwc == 23 && (rpl == 4 || rpl == 8));
  if (!ok) return fail(SJ_ERR_INVALID_ARGUMENT, "%u consumer warps x %u rows per lane not built", nwc, rpl);
  if (g.stages < 2 || g.stages > 16) return fail(SJ_ERR_INVALID_ARGUMENT, "stages=%u (2..16)", g.stages);
  if (g.chunk_rows == 0 || g.chunk_rows % (nwc * 32 * rpl) || g.chunk_rows * 4u > (1u << 19))
    return fail(SJ_ERR_INVALID_ARGUMENT, "chunk_rows=%u", g.chunk_rows);
  if (g.q1_cap < 2 * 32 * rpl || (g.q1_cap & (g.q1_cap - 1)) || g.q2_cap < 64 || (g.q2_cap & (g.q2_cap - 1)))
    return fail(SJ_ERR_INVALID_ARGUMENT, "queue capacities");
  if (g.reorder_period < 2 * g.stages) g.reorder_period = 2 * g.stages;
  g.smem_bytes = probe_smem_bytes(g);
  if (g.smem_bytes > eng->smem_optin)
    return fail(SJ_ERR_INVALID_ARGUMENT, "probe needs %u B shared memory (limit %zu)", g.smem_bytes, eng->smem_optin);
  return SJ_OK;
}

extern "C" sj_status sj_query_prepare(sj_engine* eng, const sj_plan* plan, sj_query** out) {
  if (!eng || !out) return fail(SJ_ERR_INVALID_ARGUMENT, "NULL engine/out");
  *out = nullptr;
  sj_status st = validate_plan(plan);
  if (st != SJ_OK) return st;
  SJ_CUDA(cudaSetDevice(eng->device));
  sj_query* q = new sj_query();
  q->eng = eng;
  q->plan = *plan;
  sj_plan& p = q->plan;
  if (p.row_end < 0) p.row_end = p.fact_rows;
  const bool bf_auto = p.bf_bits_per_key == SJ_BF_AUTO;
  const uint32_t bpk = bf_auto ? 0u : (uint32_t)p.bf_bits_per_key;  // auto: sized as the direct bitmap
  default_geom(eng, &p, q->geom, q->rows_per_thread);
  if (p.tune.compact_threshold) { /* compaction rounds always use full CTAs */ }
  st = check_geom(eng, q->geom, q->rows_per_thread);
  if (st != SJ_OK) {
    delete q;
    return st;
  }

  // ---- arena layout: zeroed region first (the descriptor and payload bitmaps,
  // cleared by every build's memset; the hash tables and filters, cleared by the
  // scan kernel; the group sums, left zero by the compaction kernel), then
  // uploaded / written-once data
  size_t off = 0;
  const size_t desc_off = off;
  off = align256(off + sizeof(SjDesc));
  size_t ht_off[SJ_MAX_DIMS], bf_off[SJ_MAX_DIMS], pbm_off[SJ_MAX_DIMS], inbm_off[SJ_MAX_DIMS],
      dict_off[SJ_MAX_DIMS], qual_off[SJ_MAX_DIMS];
  uint32_t bf_max_log2[SJ_MAX_DIMS];
  uint64_t groups = 1;
  for (int d = 0; d < p.n_dims; ++d) {
    const sj_dim& D = p.dims[d];
    pbm_off[d] = off;
    if (D.group) {
      const uint64_t span = (uint64_t)((int64_t)D.payload_max - D.payload_min + 1);
      off = align256(off + 4 * ((span + 31) / 32));
      groups *= span;
    }
  }
  q->head_bytes = off;
  const size_t tables_off = off;
  for (int d = 0; d < p.n_dims; ++d) {
    const sj_dim& D = p.dims[d];
    ht_off[d] = off;
    off = align256(off + sizeof(int2) * (size_t)D.ht_len);
    size_t bf_bytes;
    if (bpk == 0) {
      bf_max_log2[d] = ceil_log2((uint64_t)D.ht_len);  // bits, as roundUpToPowerOfTwo(len)
      if (bf_max_log2[d] < 6) bf_max_log2[d] = 6;
      bf_bytes = ((size_t)1 << bf_max_log2[d]) / 8;
    } else {
      const uint64_t cap_rows = (uint64_t)std::max<int64_t>(D.rows, 1);
      bf_max_log2[d] = bf_blocked_log2(cap_rows, bpk, 28);
      bf_bytes = (size_t)8 << bf_max_log2[d];
    }
    bf_off[d] = off;
    off = align256(off + std::max<size_t>(bf_bytes, 16));
  }
  const size_t tables_bytes = off - tables_off;
  q->group_capacity = groups;
  const size_t gsum_off = off;
  off = align256(off + 8 * groups);
  const size_t gcnt_off = off;
  off = align256(off + 8 * groups);
  q->zero_bytes = off;
  for (int d = 0; d < p.n_dims; ++d) {
    const sj_dim& D = p.dims[d];
    inbm_off[d] = off;
    off = align256(off + 4 * (SJ_MAX_IN_CODES / 32));
    dict_off[d] = off;
    if (D.group) off = align256(off + 4 * (size_t)((int64_t)D.payload_max - D.payload_min + 1));
    qual_off[d] = off;
    off = align256(off + 4 * (size_t)std::max<int64_t>(D.rows, 1));
  }
  const size_t rows_off = off;
  off = align256(off + sizeof(sj_group_row) * groups);
  q->arena_bytes = off;

  cudaError_t e = cudaMallocFromPoolAsync((void**)&q->arena, q->arena_bytes, eng->pool, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    const size_t bytes = q->arena_bytes;
    delete q;
    return fail(e == cudaErrorMemoryAllocation ? SJ_ERR_OUT_OF_MEMORY : SJ_ERR_CUDA, "query arena of %zu B: %s", bytes,
                cudaGetErrorString(e));
  }

  // hash tables and filters lie in [tables_off, tables_off + tables_bytes) of the arena
  q->l2win = l2_window(q->arena + tables_off, tables_bytes, eng->l2_persist_bytes, eng->l2_window_max);

  // ---- runtime parameters
  SjPlanRt& rt = q->rt;
  memset(&rt, 0, sizeof(rt));
  rt.desc = reinterpret_cast<SjDesc*>(q->arena + desc_off);
  rt.zero_tables = q->arena + tables_off;
  rt.zero_tables_bytes = tables_bytes;
  rt.measure = p.measure;
  rt.measure_sub = p.measure_sub;
  rt.g_sum = reinterpret_cast<unsigned long long*>(q->arena + gsum_off);
  rt.g_cnt = reinterpret_cast<unsigned long long*>(q->arena + gcnt_off);
  rt.rows_out = reinterpret_cast<sj_group_row*>(q->arena + rows_off);
  rt.row_begin = (uint64_t)p.row_begin;
  rt.row_end = (uint64_t)p.row_end;
  rt.n_dims = (uint32_t)p.n_dims;
  rt.lip = p.lip ? 1u : 0u;
  rt.adaptive = p.adaptive ? 1u : 0u;
  rt.group_capacity = (uint32_t)groups;
  rt.bf_smem_budget = q->geom.bf_smem_bytes;
  for (int i = 0; i < SJ_MAX_DIMS; ++i) rt.order[i] = (i < p.n_dims) ? (uint32_t)p.order[i] : 0u;
  q->in_bitmaps.assign(SJ_MAX_DIMS * (SJ_MAX_IN_CODES / 32), 0u);
  for (int d = 0; d < p.n_dims; ++d) {
    const sj_dim& D = p.dims[d];
    SjDimRt& R = rt.dim[d];
    R.fact_fk = D.fact_fk;
    R.key = D.key;
    R.filter_attr = D.filter_attr;
    R.payload = D.payload;
    R.in_bitmap = reinterpret_cast<const uint32_t*>(q->arena + inbm_off[d]);
    R.ht = reinterpret_cast<int2*>(q->arena + ht_off[d]);
    R.bf = q->arena + bf_off[d];
    R.payload_bitmap = reinterpret_cast<uint32_t*>(q->arena + pbm_off[d]);
    R.dict = reinterpret_cast<int32_t*>(q->arena + dict_off[d]);
    R.qual_rows = reinterpret_cast<uint32_t*>(q->arena + qual_off[d]);
    R.rows = (uint64_t)D.rows;
    R.fastmod_m = ~0ull / (uint64_t)(uint32_t)D.ht_len + 1ull;
    R.key_min = D.key_min;
    R.ht_len = (uint32_t)D.ht_len;
    R.pred_kind = D.pred_kind;
    R.pred_lo = D.pred_lo;
    R.pred_hi = D.pred_hi;
    R.payload_min = D.payload_min;
    R.payload_span = D.group ? (uint32_t)((int64_t)D.payload_max - D.payload_min + 1) : 0u;
    R.grouped = D.group ? 1u : 0u;
    R.bf_mode = bf_auto ? kBfAuto : (bpk ? kBfBlocked : kBfDirect);
    R.bf_k = (bpk || bf_auto) ? (uint32_t)p.bf_hashes : 1u;
    R.bf_bits_per_key = bf_auto ? kAutoBitsPerKey : bpk;
    R.bf_max_log2 = bf_max_log2[d];
    if (D.pred_kind == SJ_PRED_IN) {
      uint32_t* bm = q->in_bitmaps.data() + d * (SJ_MAX_IN_CODES / 32);
      for (int i = 0; i < D.in_count; ++i) bm[D.in_codes[i] >> 5] |= 1u << (D.in_codes[i] & 31);
    }
  }
  for (int d = 0; d < p.n_dims; ++d) {
    e = cudaMemcpy(q->arena + inbm_off[d], q->in_bitmaps.data() + d * (SJ_MAX_IN_CODES / 32),
                   4 * (SJ_MAX_IN_CODES / 32), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFreeAsync(q->arena, 0);
      delete q;
      return fail(SJ_ERR_CUDA, "uploading IN-list bitmaps: %s", cudaGetErrorString(e));
    }
  }
  cudaEventCreate(&q->ev_start);
  cudaEventCreate(&q->ev_built);
  cudaEventCreate(&q->ev_probed);
  *out = q;
  return SJ_OK;
}

extern "C" sj_status sj_query_build(sj_query* q, void* stream) {
  SjNvtxRange nvtx_range("sj.query.build");
  if (!q) return fail(SJ_ERR_INVALID_ARGUMENT, "NULL query");
  cudaStream_t st = (cudaStream_t)stream;
  SJ_CUDA(cudaSetDevice(q->eng->device));
  const bool events = q->plan.tune.record_events != 0;
  if (events) SJ_CUDA(cudaEventRecord(q->ev_start, st));
  // the scan kernel clears the hash tables and filters, the compaction kernel
  // leaves the group sums zero; the whole region is cleared only after prepare
  // and after an error
  const bool head_only = q->groups_clean;
  if (head_only) {  // a kernel, so the scan can be its programmatic dependent
    const uint64_t n16 = q->head_bytes / 16;
    const uint32_t blocks = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n16 + 255) / 256, 64));
    sj_clear_head<<<blocks, 256, 0, st>>>(reinterpret_cast<uint4*>(q->arena), n16);
    SJ_CUDA(cudaGetLastError());
  } else {
    SJ_CUDA(cudaMemsetAsync(q->arena, 0, q->zero_bytes, st));
  }
  q->groups_clean = true;
  int64_t max_rows = 1;
  uint32_t max_pwords = 1;
  for (int d = 0; d < q->plan.n_dims; ++d) {
    max_rows = std::max<int64_t>(max_rows, q->plan.dims[d].rows);
    max_pwords = std::max<uint32_t>(max_pwords, (q->rt.dim[d].payload_span + 31) / 32);
  }
  uint32_t bx = (uint32_t)std::min<int64_t>((max_rows + 255) / 256, (int64_t)q->eng->sm_count * 8);
  if (bx < 1) bx = 1;
  dim3 grid(bx, (unsigned)q->plan.n_dims);
  SJ_CUDA(launch_windowed(sj_dim_scan, grid, dim3(256), 0, st, L2Window{}, head_only, q->rt));
  // the insert walks only the listed qualifying rows: a smaller grid
  const dim3 igrid(std::max(1u, std::min<uint32_t>(bx, (uint32_t)q->eng->sm_count * 2)), (unsigned)q->plan.n_dims);
  SJ_CUDA(launch_windowed(sj_dim_insert, igrid, dim3(256), 4 * max_pwords, st, L2Window{}, true, q->rt));
  if (events) SJ_CUDA(cudaEventRecord(q->ev_built, st));
  q->built = true;
  q->probed_since_build = false;
  q->stream = st;
  return SJ_OK;
}

extern "C" sj_status sj_query_probe(sj_query* q, void* stream) {
  SjNvtxRange nvtx_range("sj.query.probe");
  if (!q) return fail(SJ_ERR_INVALID_ARGUMENT, "NULL query");
  if (!q->built) return fail(SJ_ERR_INVALID_ARGUMENT, "probe before build");
  cudaStream_t st = (cudaStream_t)stream;
  SJ_CUDA(cudaSetDevice(q->eng->device));
  const bool again = q->probed_since_build;
  if (again) {  // probe again over the same build: counters and result rows start over
    const size_t first = offsetof(SjDesc, groups_out);
    SJ_CUDA(cudaMemsetAsync(reinterpret_cast<uint8_t*>(q->rt.desc) + first, 0, sizeof(SjDesc) - first, st));
  }
  q->probed_since_build = true;
  if (q->rt.row_end > q->rt.row_begin) {
    q->groups_clean = false;  // until the compaction kernel has cleared them again
    SJ_CUDA(launch_probe(q->rt, q->geom, q->rows_per_thread, st, q->l2win, !again));  // after the insert kernel
  }
  SJ_CUDA(launch_finalize(q->rt, (uint32_t)q->group_capacity, st, true));
  q->groups_clean = true;
  if (q->plan.tune.record_events) SJ_CUDA(cudaEventRecord(q->ev_probed, st));
  q->probed = true;
  q->stream = st;
  return SJ_OK;
}

static bool row_less(const sj_group_row& a, const sj_group_row& b) {
  for (int d = 0; d < SJ_MAX_DIMS; ++d)
    if (a.attr[d] != b.attr[d]) return a.attr[d] < b.attr[d];
  return false;
}

extern "C" sj_status sj_query_fetch(sj_query* q, sj_group_row* out, int64_t cap, int64_t* n_out, void* stream) {
  SjNvtxRange nvtx_range("sj.query.fetch");
  if (!q || !n_out) return fail(SJ_ERR_INVALID_ARGUMENT, "NULL query/n_out");
  if (!q->probed) return fail(SJ_ERR_INVALID_ARGUMENT, "fetch before probe");
  cudaStream_t st = (cudaStream_t)stream;
  SJ_CUDA(cudaSetDevice(q->eng->device));
  SjDesc desc;
  SJ_CUDA(cudaMemcpyAsync(&desc, q->rt.desc, sizeof(desc), cudaMemcpyDeviceToHost, st));
  SJ_CUDA(cudaStreamSynchronize(st));
  if (desc.error_flags) q->groups_clean = false;
  if (desc.error_flags & kErrWaitTimeout) return fail(SJ_ERR_TIMEOUT, "probe kernel: bounded wait expired");
  if (desc.error_flags & kErrPayloadDomain)
    return fail(SJ_ERR_INVALID_ARGUMENT, "a grouped payload lies outside [payload_min, payload_max]");
  if (desc.error_flags) return fail(SJ_ERR_CUDA, "device error flags 0x%x", desc.error_flags);
  const int64_t n = desc.groups_out;
  *n_out = n;
  if (n > cap || (n > 0 && !out)) return fail(SJ_ERR_CAPACITY, "need %lld result rows", (long long)n);
  if (n > 0) {
    SJ_CUDA(cudaMemcpyAsync(out, q->rt.rows_out, sizeof(sj_group_row) * (size_t)n, cudaMemcpyDeviceToHost, st));
    SJ_CUDA(cudaStreamSynchronize(st));
    std::sort(out, out + n, row_less);
  }
  return SJ_OK;
}

extern "C" sj_status sj_query_get_stats(sj_query* q, sj_query_stats* out) {
  if (!q || !out) return fail(SJ_ERR_INVALID_ARGUMENT, "NULL query/out");
  SJ_CUDA(cudaSetDevice(q->eng->device));
  SJ_CUDA(cudaStreamSynchronize(q->stream));
  SjDesc desc;
  SJ_CUDA(cudaMemcpy(&desc, q->rt.desc, sizeof(desc), cudaMemcpyDeviceToHost));
  memset(out, 0, sizeof(*out));
  out->rows_scanned = desc.rows_scanned;
  for (int i = 0; i < 2 * SJ_MAX_DIMS; ++i) {
    out->step_in[i] = desc.step_in[i];
    out->step_out[i] = desc.step_out[i];
  }
  for (int d = 0; d < q->plan.n_dims; ++d) {
    out->bf_inserted[d] = desc.dim[d].n_inserted;
    const uint32_t l2 = desc.dim[d].bf_log2;
    out->bf_words[d] = desc.dim[d].bf_mode == kBfDirect ? std::max<uint64_t>(2, (1ull << l2) / 32) : (2ull << l2);
    out->bf_blocked[d] = desc.dim[d].bf_mode == kBfBlocked ? 1 : 0;
  }
  out->groups = desc.groups_out;
  out->reorders = desc.reorders;
  out->error_flags = desc.error_flags;
  float ms = 0.f;
  if (q->plan.tune.record_events) {
    if (q->built && cudaEventElapsedTime(&ms, q->ev_start, q->ev_built) == cudaSuccess) out->build_ms = ms;
    if (q->probed && cudaEventElapsedTime(&ms, q->ev_built, q->ev_probed) == cudaSuccess) out->probe_ms = ms;
  }
  cudaGetLastError();
  return SJ_OK;
}

extern "C" void sj_query_release(sj_query* q) {
  if (!q) return;
  cudaSetDevice(q->eng->device);
  if (q->arena) cudaFreeAsync(q->arena, q->stream);
  if (q->ev_start) cudaEventDestroy(q->ev_start);
  if (q->ev_built) cudaEventDestroy(q->ev_built);
  if (q->ev_probed) cudaEventDestroy(q->ev_probed);
  delete q;
}

// ------------------------------------------------------------ run plain ----
namespace {
// Device copies of host columns for sj_run_plain(host_columns = 1).
struct Staging {
  std::vector<std::pair<const int32_t*, int32_t*>> map;
  cudaMemPool_t pool;
  cudaStream_t st;
  ~Staging() {
    for (auto& m : map) cudaFreeAsync(m.second, st);
  }
  cudaError_t get(const int32_t* host, int64_t n, const int32_t** dev) {
    if (!host) {
      *dev = nullptr;
      return cudaSuccess;
    }
    for (auto& m : map)
      if (m.first == host) {
        *dev = m.second;
        return cudaSuccess;
      }
    int32_t* d = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync((void**)&d, std::max<size_t>(16, 4 * (size_t)n), pool, st);
    if (e != cudaSuccess) return e;
    map.push_back({host, d});
    if (n > 0) e = cudaMemcpyAsync(d, host, 4 * (size_t)n, cudaMemcpyHostToDevice, st);
    *dev = d;
    return e;
  }
};
}  // namespace

// Device address of a column a kernel may read directly: device memory, managed
// memory, or pinned host memory mapped into the device's address space.
static bool device_readable(const void* p, const int32_t** dev) {
  if (!p) {
    *dev = nullptr;
    return true;
  }
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if ((a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) &&
      a.devicePointer) {
    *dev = reinterpret_cast<const int32_t*>(a.devicePointer);
    return true;
  }
  return false;
}

static sj_status run_query_whole(sj_engine* eng, const sj_plan& p, sj_group_row* out, int64_t cap, int64_t* n_out,
                                 cudaStream_t st, cudaEvent_t t1) {
  sj_query* q = nullptr;
  sj_status s = sj_query_prepare(eng, &p, &q);
  if (s == SJ_OK) s = sj_query_build(q, st);
  if (s == SJ_OK) s = sj_query_probe(q, st);
  cudaEventRecord(t1, st);
  if (s == SJ_OK) s = sj_query_fetch(q, out, cap, n_out, st);
  if (q) sj_query_release(q);
  return s;
}

// Host-column query: the dimension tables are copied to the device; the fact
// column tested first streams to the device in pieces on a second stream,
// overlapped with probe launches over the pieces already present (group
// partials accumulate across launches); the other fact columns stay in pinned
// host memory and are read in place at survivor rows only.
static sj_status run_query_streamed(sj_engine* eng, sj_plan p, const int32_t* host_first, sj_group_row* out,
                                    int64_t cap, int64_t* n_out, cudaStream_t st, cudaEvent_t t1) {
  SjNvtxRange nvtx_range("sj.run_plain.streamed");
  const int first = p.order[0];
  const int64_t b = p.row_begin, e = p.row_end;
  const int64_t base = b & ~3ll;
  int32_t* dev = nullptr;
  SJ_CUDA(cudaMallocFromPoolAsync((void**)&dev, std::max<size_t>(16, 4 * (size_t)p.fact_rows), eng->pool, st));
  p.dims[first].fact_fk = dev;
  p.adaptive = 0;  // the streamed column is fixed; the others are host-resident
  sj_query* q = nullptr;
  sj_status s = sj_query_prepare(eng, &p, &q);
  cudaStream_t cs = nullptr;
  std::vector<cudaEvent_t> evs;
  if (s == SJ_OK) s = sj_query_build(q, st);
  if (s == SJ_OK) {
    cs = eng->copy_stream;
    cudaEvent_t ready;
    cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    cudaEventRecord(ready, st);  // the allocation is ordered on st
    cudaStreamWaitEvent(cs, ready, 0);
    evs.push_back(ready);
    const int64_t span = e - base;
    const int64_t pieces = std::max<int64_t>(1, std::min<int64_t>(8, span / (1ll << 20)));
    int64_t pb = base;
    for (int64_t i = 0; i < pieces && s == SJ_OK; ++i) {
      int64_t pe = (i + 1 == pieces) ? e : ((base + span * (i + 1) / pieces) & ~3ll);
      if (pe <= pb) continue;
      cudaError_t ce = cudaMemcpyAsync(dev + pb, host_first + pb, 4 * (size_t)(pe - pb), cudaMemcpyHostToDevice, cs);
      cudaEvent_t ev;
      cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      cudaEventRecord(ev, cs);
      evs.push_back(ev);
      cudaStreamWaitEvent(st, ev, 0);
      SjPlanRt rt = q->rt;
      rt.row_begin = (uint64_t)std::max<int64_t>(pb, b);
      rt.row_end = (uint64_t)pe;
      if (ce == cudaSuccess) ce = launch_probe(rt, q->geom, q->rows_per_thread, st, q->l2win, false);
      if (ce != cudaSuccess) s = fail(SJ_ERR_CUDA, "streamed probe: %s", cudaGetErrorString(ce));
      pb = pe;
    }
  }
  if (s == SJ_OK) {
    cudaError_t ce = launch_finalize(q->rt, (uint32_t)q->group_capacity, st, false);
    if (ce != cudaSuccess) s = fail(SJ_ERR_CUDA, "finalize: %s", cudaGetErrorString(ce));
    q->built = q->probed = true;
    q->stream = st;
  }
  cudaEventRecord(t1, st);
  if (s == SJ_OK) s = sj_query_fetch(q, out, cap, n_out, st);
  cudaStreamSynchronize(st);
  for (cudaEvent_t ev : evs) cudaEventDestroy(ev);
  if (q) sj_query_release(q);
  cudaFreeAsync(dev, st);
  return s;
}

extern "C" sj_status sj_run_plain(sj_engine* eng, const sj_plan* plan, int host_columns, sj_group_row* out,
                                  int64_t cap, int64_t* n_out, float* ms, void* stream) {
  SjNvtxRange nvtx_range("sj.run_plain");
  if (!eng || !plan || !n_out) return fail(SJ_ERR_INVALID_ARGUMENT, "NULL engine/plan/n_out");
  cudaStream_t st = (cudaStream_t)stream;
  SJ_CUDA(cudaSetDevice(eng->device));
  sj_status s = validate_plan(plan);
  if (s != SJ_OK) return s;
  sj_plan p = *plan;
  if (p.row_end < 0) p.row_end = p.fact_rows;
  Staging stg;
  stg.pool = eng->pool;
  stg.st = st;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, st);
  if (!host_columns) {
    s = run_query_whole(eng, p, out, cap, n_out, st, t1);
  } else {
    // dimension tables: small, copied
    cudaError_t e = cudaSuccess;
    for (int d = 0; d < p.n_dims && e == cudaSuccess; ++d) {
      sj_dim& D = p.dims[d];
      e = stg.get(plan->dims[d].key, D.rows, &D.key);
      if (e == cudaSuccess) e = stg.get(plan->dims[d].filter_attr, D.rows, &D.filter_attr);
      if (e == cudaSuccess) e = stg.get(plan->dims[d].payload, D.rows, &D.payload);
    }
    // fact columns: read in place when the device can address them (pinned)
    bool mapped = true;
    for (int d = 0; d < p.n_dims; ++d) mapped = mapped && device_readable(plan->dims[d].fact_fk, &p.dims[d].fact_fk);
    mapped = mapped && device_readable(plan->measure, &p.measure) &&
             device_readable(plan->measure_sub, &p.measure_sub);
    if (e == cudaSuccess && mapped) {
      s = run_query_streamed(eng, p, plan->dims[p.order[0]].fact_fk, out, cap, n_out, st, t1);
    } else if (e == cudaSuccess) {
      // pageable host memory: stage every fact column
      const int64_t fr = p.fact_rows;
      for (int d = 0; d < p.n_dims && e == cudaSuccess; ++d) e = stg.get(plan->dims[d].fact_fk, fr, &p.dims[d].fact_fk);
      if (e == cudaSuccess) e = stg.get(plan->measure, fr, &p.measure);
      if (e == cudaSuccess) e = stg.get(plan->measure_sub, fr, &p.measure_sub);
      if (e == cudaSuccess) s = run_query_whole(eng, p, out, cap, n_out, st, t1);
    }
    if (e != cudaSuccess)
      s = fail(e == cudaErrorMemoryAllocation ? SJ_ERR_OUT_OF_MEMORY : SJ_ERR_CUDA, "staging host columns: %s",
               cudaGetErrorString(e));
  }
  if (ms) {
    cudaEventSynchronize(t1);
    float v = 0.f;
    if (cudaEventElapsedTime(&v, t0, t1) == cudaSuccess) *ms = v;
    cudaGetLastError();
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  return s;
}

// --------------------------------------------------------- SSB Q3.3 call ----
extern "C" sj_status sj_ssb_q33_run(sj_engine* e, const int32_t* lo_orderdate, const int32_t* lo_custkey,
                                    const int32_t* lo_suppkey, const int32_t* lo_revenue, int64_t lo_len,
                                    const int32_t* d_datekey, const int32_t* d_year, int64_t d_len,
                                    const int32_t* s_suppkey, const int32_t* s_city, int64_t s_len,
                                    const int32_t* c_custkey, const int32_t* c_city, int64_t c_len,
                                    const int32_t order[3], int32_t lip, int32_t bf_bits_per_key, sj_group_row* out,
                                    int64_t cap, int64_t* n_out, float* time_query_ms) {
  static const int32_t kCities[2] = {231, 235};  // src/ssb-jo/q33/0-lip.cu:132-135
  if (!order) return fail(SJ_ERR_INVALID_ARGUMENT, "order is NULL");
  sj_plan p;
  memset(&p, 0, sizeof(p));
  p.n_dims = 3;
  // dim 0 = supplier
  p.dims[0] = sj_dim{lo_suppkey, s_suppkey, s_city, s_city, s_len, 0, (int32_t)s_len, SJ_PRED_IN, 0, 0, 2,
                     kCities, 1, 0, 249};
  // dim 1 = customer
  p.dims[1] = sj_dim{lo_custkey, c_custkey, c_city, c_city, c_len, 0, (int32_t)c_len, SJ_PRED_IN, 0, 0, 2,
                     kCities, 1, 0, 249};
  // dim 2 = date: d_year <= 1997 (BlockPredGTE(1992) is overwritten by BlockPredLTE(1997),
  // src/ssb-jo/q33/0-lip.cu:187-190); key-range table of 19981230-19920101+1 slots (:219)
  p.dims[2] = sj_dim{lo_orderdate, d_datekey, d_year, d_year, d_len, 19920101, 19981230 - 19920101 + 1,
                     SJ_PRED_RANGE, INT32_MIN, 1997, 0, nullptr, 1, 1992, 1998};
  p.measure = lo_revenue;
  p.fact_rows = lo_len;
  p.row_begin = 0;
  p.row_end = lo_len;
  for (int i = 0; i < 3; ++i) p.order[i] = order[i];
  p.lip = lip;
  p.adaptive = 0;
  p.bf_bits_per_key = bf_bits_per_key;
  p.bf_hashes = bf_bits_per_key ? 2 : 1;
  return sj_run_plain(e, &p, 0, out, cap, n_out, time_query_ms, nullptr);
}

// -------------------------------------------------------- Bloom unit test ----
__global__ void sj_bloom_build_kernel(const int32_t* keys, const int32_t* flags, int64_t n, void* bf, uint32_t mode,
                                      uint32_t log2, uint32_t k, int32_t kmin) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (flags && !flags[i]) continue;
    const uint32_t s = (uint32_t)keys[i] - (uint32_t)kmin;
    if (mode == kBfDirect) {
      const uint32_t b = s & ((1u << log2) - 1u);
      atomicOr(reinterpret_cast<uint32_t*>(bf) + (b >> 5), 1u << (b & 31u));
    } else {
      atomicOr(reinterpret_cast<unsigned long long*>(bf) + bf_word(s, log2),
               (unsigned long long)bf_mask(s, k));
    }
  }
}

__global__ void sj_bloom_probe_kernel(const int32_t* keys, int64_t n, int32_t* out, const void* bf, uint32_t mode,
                                      uint32_t log2, uint32_t k, int32_t kmin) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t s = (uint32_t)keys[i] - (uint32_t)kmin;
    int32_t hit;
    if (mode == kBfDirect) {
      const uint32_t b = s & ((1u << log2) - 1u);
      hit = (reinterpret_cast<const uint32_t*>(bf)[b >> 5] >> (b & 31u)) & 1u;
    } else {
      const uint64_t m = bf_mask(s, k);
      hit = (reinterpret_cast<const unsigned long long*>(bf)[bf_word(s, log2)] & m) == m;
    }
    out[i] = hit;
  }
}

extern "C" sj_status sj_bloom_test(const int32_t* keys, const int32_t* flags, int64_t n_keys,
                                   const int32_t* probe_keys, int32_t* out_flags, int64_t n_probe,
                                   int32_t bits_per_key, int32_t hashes, int32_t key_min, int32_t direct_words,
                                   void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n_keys < 0 || n_probe < 0 || (n_keys && !keys) || (n_probe && (!probe_keys || !out_flags)))
    return fail(SJ_ERR_INVALID_ARGUMENT, "bad buffers");
  uint32_t mode, log2, k;
  size_t bytes;
  if (bits_per_key == 0) {
    if (direct_words < 1 || (direct_words & (direct_words - 1)))
      return fail(SJ_ERR_INVALID_ARGUMENT, "direct_words must be a power of two");
    mode = kBfDirect;
    log2 = ceil_log2((uint64_t)direct_words * 32);
    k = 1;
    bytes = (size_t)direct_words * 4;
  } else {
    if (hashes < 1 || hashes > 4) return fail(SJ_ERR_INVALID_ARGUMENT, "hashes 1..4");
    mode = kBfBlocked;
    // size by the number of keys that will be inserted
    int64_t n_ins = n_keys;
    if (flags) {
      std::vector<int32_t> hf((size_t)n_keys);
      SJ_CUDA(cudaMemcpy(hf.data(), flags, 4 * (size_t)n_keys, cudaMemcpyDeviceToHost));
      n_ins = 0;
      for (int32_t f : hf) n_ins += f != 0;
    }
    log2 = bf_blocked_log2((uint64_t)n_ins, (uint32_t)bits_per_key, 28);
    k = (uint32_t)hashes;
    bytes = (size_t)8 << log2;
  }
  void* bf = nullptr;
  SJ_CUDA(cudaMalloc(&bf, bytes));
  cudaMemsetAsync(bf, 0, bytes, st);
  if (n_keys) sj_bloom_build_kernel<<<256, 256, 0, st>>>(keys, flags, n_keys, bf, mode, log2, k, key_min);
  if (n_probe) sj_bloom_probe_kernel<<<256, 256, 0, st>>>(probe_keys, n_probe, out_flags, bf, mode, log2, k, key_min);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(bf);
  if (e != cudaSuccess) return fail(SJ_ERR_CUDA, "bloom test: %s", cudaGetErrorString(e));
  return SJ_OK;
}

// ------------------------------------------------------------ generators ----
__global__ void sj_gen_kernel(int32_t* dst, int64_t n, uint64_t row0, uint64_t key, int32_t kind, int32_t lo,
                              int32_t hi) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = sj_gen_value(key, kind, lo, hi, row0 + (uint64_t)i);
}

extern "C" sj_status sj_gen_rows_device(int32_t* dst, int64_t row0, int64_t n, uint64_t seed, int32_t col,
                                        int32_t kind, int32_t lo, int32_t hi, void* stream) {
  if (n < 0 || row0 < 0 || (n && !dst)) return fail(SJ_ERR_INVALID_ARGUMENT, "bad buffer");
  if (n == 0) return SJ_OK;
  sj_gen_kernel<<<1184, 256, 0, (cudaStream_t)stream>>>(dst, n, (uint64_t)row0, sj_stream_key(seed, (uint32_t)col),
                                                        kind, lo, hi);
  SJ_CUDA(cudaGetLastError());
  return SJ_OK;
}

extern "C" sj_status sj_gen_column_device(int32_t* dst, int64_t n, uint64_t seed, int32_t col, int32_t kind,
                                          int32_t lo, int32_t hi, void* stream) {
  return sj_gen_rows_device(dst, 0, n, seed, col, kind, lo, hi, stream);
}

// Host generator (no GPU needed): same values as sj_gen_column_device.
extern "C" void sj_gen_column_host(int32_t* dst, int64_t n, uint64_t seed, int32_t col, int32_t kind, int32_t lo,
                                   int32_t hi, int threads) {
  const uint64_t key = sj_stream_key(seed, (uint32_t)col);
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  if (n < 1 << 16) threads = 1;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    const int64_t b = n * t / threads, e = n * (t + 1) / threads;
    auto work = [=]() {
      for (int64_t i = b; i < e; ++i) dst[i] = sj_gen_value(key, kind, lo, hi, (uint64_t)i);
    };
    if (t + 1 == threads) work();
    else pool.emplace_back(work);
  }
  for (auto& th : pool) th.join();
}
