// sj_noalloc.cu -- the Q3.3 star join without any device allocation.
//
// Some callers cannot allocate device memory during a query: an application
// that runs inside a fixed device-memory budget handed out up front, a host that
// forbids allocator calls on its latency path (cudaMalloc can synchronize the
// device and stall unrelated work), or an embedding runtime that owns every
// allocation itself.  sj_ssb_q33_run_noalloc serves them: it runs the same
// build / probe / finalize kernels as sj_ssb_q33_run, but every byte of scratch
// (hash tables, filters, group partials, result rows) lives in one file-scope
// device array of fixed size, reserved when the library is loaded and held by
// every GPU that loads it until the process exits.  The caller passes the input
// columns (device memory) and the host buffer that receives the result rows.
//
// The array is shared by every call on a device and keeps the previous call's
// contents; each call clears the parts that must start at zero.  Calls that
// overlap on the GPU (different streams or host threads at the same time) race
// on the array and must be serialized by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "sj_internal.h"

namespace sj {
uint32_t probe_smem_bytes(const SjProbeGeom& g);
cudaError_t launch_probe(const SjPlanRt& P, const SjProbeGeom& G, uint32_t rows_per_thread, cudaStream_t st,
                         const L2Window& w, bool pdl);
cudaError_t launch_finalize(const SjPlanRt& P, uint32_t group_capacity, cudaStream_t st, bool pdl);
__global__ void sj_dim_scan(const __grid_constant__ SjPlanRt P);
__global__ void sj_dim_insert(const __grid_constant__ SjPlanRt P);
}  // namespace sj

using namespace sj;

// Scratch of the no-allocation entry point: 48 MiB per device.
#define SJ_NOALLOC_SCRATCH_BYTES (48ull << 20)
static __device__ __align__(256) unsigned char sj_noalloc_scratch[SJ_NOALLOC_SCRATCH_BYTES];

static thread_local std::string g_noalloc_error;
extern "C" const char* sj_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

static sj_status na_fail(sj_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_noalloc_error = buf;
  return s;
}

// Device address of the scratch array in the current device's context (the
// host-side symbol itself is not a device address).  Looked up on every call,
// with the call's device current: the lookup allocates nothing, and an address
// cached across calls would go stale when the caller resets the device
// (cudaDeviceReset) and the library's device code is loaded into a new context.
static sj_status scratch_address(int device, unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, sj_noalloc_scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return na_fail(SJ_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", device, cudaGetErrorString(e));
  }
  *out = static_cast<unsigned char*>(p);
  return SJ_OK;
}

static size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" sj_status sj_ssb_q33_run_noalloc(int device, const int32_t* lo_orderdate, const int32_t* lo_custkey,
                                            const int32_t* lo_suppkey, const int32_t* lo_revenue, int64_t lo_len,
                                            const int32_t* d_datekey, const int32_t* d_year, int64_t d_len,
                                            const int32_t* s_suppkey, const int32_t* s_city, int64_t s_len,
                                            const int32_t* c_custkey, const int32_t* c_city, int64_t c_len,
                                            const int32_t order[3], int32_t lip, int32_t bf_bits_per_key,
                                            sj_group_row* out, int64_t cap, int64_t* n_out, void* stream) {
  const cudaStream_t st = (cudaStream_t)stream;
  if (!order || !n_out) return na_fail(SJ_ERR_INVALID_ARGUMENT, "order / n_out is NULL");
  if (!lo_orderdate || !lo_custkey || !lo_suppkey || !lo_revenue || !d_datekey || !d_year || !s_suppkey ||
      !s_city || !c_custkey || !c_city)
    return na_fail(SJ_ERR_INVALID_ARGUMENT, "NULL column");
  if (lo_len < 0 || lo_len > 0xFFFFFFF0ll || d_len <= 0 || s_len <= 0 || c_len <= 0 || s_len > INT32_MAX ||
      c_len > INT32_MAX || d_len > INT32_MAX)
    return na_fail(SJ_ERR_INVALID_ARGUMENT, "table length out of range");
  const void* fact[4] = {lo_orderdate, lo_custkey, lo_suppkey, lo_revenue};
  for (const void* f : fact)
    if (reinterpret_cast<uintptr_t>(f) & 15u) return na_fail(SJ_ERR_INVALID_ARGUMENT, "fact column not 16-byte aligned");
  int used[3] = {0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    if (order[i] < 0 || order[i] > 2 || used[order[i]]) return na_fail(SJ_ERR_INVALID_ARGUMENT, "order");
    used[order[i]] = 1;
  }
  if (bf_bits_per_key < 0 || bf_bits_per_key > 64) return na_fail(SJ_ERR_INVALID_ARGUMENT, "bf_bits_per_key");

  // dims: 0 supplier, 1 customer, 2 date (as sj_ssb_q33_run, src/ssb-jo/q33/0-lip.cu:114-203)
  const int64_t rows[3] = {s_len, c_len, d_len};
  const uint32_t ht_len[3] = {(uint32_t)s_len, (uint32_t)c_len, 19981230u - 19920101u + 1u};
  const int32_t key_min[3] = {0, 0, 19920101};
  const int32_t pmin[3] = {0, 0, 1992};
  const uint32_t span[3] = {250, 250, 7};
  const uint32_t bpk = (uint32_t)bf_bits_per_key;

  // ---- scratch layout (zeroed part first) and the size check
  size_t off = 0;
  const size_t desc_off = off;
  off = a256(off + sizeof(SjDesc));
  size_t ht_off[3], bf_off[3], pbm_off[3], inbm_off[3], dict_off[3], qual_off[3];
  uint32_t bf_log2[3];
  for (int d = 0; d < 3; ++d) {
    ht_off[d] = off;
    off = a256(off + sizeof(int2) * (size_t)ht_len[d]);
    size_t bytes;
    if (bpk == 0) {
      bf_log2[d] = std::max<uint32_t>(6, ceil_log2(ht_len[d]));
      bytes = ((size_t)1 << bf_log2[d]) / 8;
    } else {
      bf_log2[d] = bf_blocked_log2((uint64_t)rows[d], bpk, 28);
      bytes = (size_t)8 << bf_log2[d];
    }
    bf_off[d] = off;
    off = a256(off + std::max<size_t>(bytes, 16));
    pbm_off[d] = off;
    off = a256(off + 4 * ((span[d] + 31) / 32));
  }
  const uint64_t groups = 250ull * 250ull * 7ull;
  const size_t gsum_off = off;
  off = a256(off + 8 * groups);
  const size_t gcnt_off = off;
  off = a256(off + 8 * groups);
  const size_t zero_bytes = off;
  for (int d = 0; d < 3; ++d) {
    inbm_off[d] = off;
    off = a256(off + 4 * (SJ_MAX_IN_CODES / 32));
    dict_off[d] = off;
    off = a256(off + 4 * (size_t)span[d]);
    qual_off[d] = off;
    off = a256(off + 4 * (size_t)rows[d]);
  }
  const size_t rows_off = off;
  off = a256(off + sizeof(sj_group_row) * groups);
  if (off > SJ_NOALLOC_SCRATCH_BYTES)
    return na_fail(SJ_ERR_CAPACITY, "query needs %zu bytes of scratch; the no-allocation entry point has %llu", off,
                   (unsigned long long)SJ_NOALLOC_SCRATCH_BYTES);

  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return na_fail(SJ_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
  unsigned char* base = nullptr;
  sj_status s = scratch_address(device, &base);
  if (s != SJ_OK) return s;
  int sms = 0, smem_optin = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (e != cudaSuccess) return na_fail(SJ_ERR_CUDA, "device attribute: %s", cudaGetErrorString(e));

  // ---- runtime parameters
  SjPlanRt rt;
  memset(&rt, 0, sizeof(rt));
  rt.desc = reinterpret_cast<SjDesc*>(base + desc_off);
  rt.measure = lo_revenue;
  rt.g_sum = reinterpret_cast<unsigned long long*>(base + gsum_off);
  rt.g_cnt = reinterpret_cast<unsigned long long*>(base + gcnt_off);
  rt.rows_out = reinterpret_cast<sj_group_row*>(base + rows_off);
  rt.row_begin = 0;
  rt.row_end = (uint64_t)lo_len;
  rt.n_dims = 3;
  rt.lip = lip ? 1u : 0u;
  rt.adaptive = 0;
  rt.group_capacity = (uint32_t)groups;
  for (int i = 0; i < 3; ++i) rt.order[i] = (uint32_t)order[i];
  const int32_t* fks[3] = {lo_suppkey, lo_custkey, lo_orderdate};
  const int32_t* keys[3] = {s_suppkey, c_custkey, d_datekey};
  const int32_t* attrs[3] = {s_city, c_city, d_year};
  uint32_t in_bitmaps[3][SJ_MAX_IN_CODES / 32];
  memset(in_bitmaps, 0, sizeof(in_bitmaps));
  in_bitmaps[0][231 >> 5] |= 1u << (231 & 31);  // s_city IN {231, 235} (0-lip.cu:132-135)
  in_bitmaps[0][235 >> 5] |= 1u << (235 & 31);
  in_bitmaps[1][231 >> 5] |= 1u << (231 & 31);  // c_city IN {231, 235}
  in_bitmaps[1][235 >> 5] |= 1u << (235 & 31);
  for (int d = 0; d < 3; ++d) {
    SjDimRt& R = rt.dim[d];
    R.fact_fk = fks[d];
    R.key = keys[d];
    R.filter_attr = attrs[d];
    R.payload = attrs[d];
    R.in_bitmap = reinterpret_cast<const uint32_t*>(base + inbm_off[d]);
    R.ht = reinterpret_cast<int2*>(base + ht_off[d]);
    R.bf = base + bf_off[d];
    R.payload_bitmap = reinterpret_cast<uint32_t*>(base + pbm_off[d]);
    R.dict = reinterpret_cast<int32_t*>(base + dict_off[d]);
    R.qual_rows = reinterpret_cast<uint32_t*>(base + qual_off[d]);
    R.rows = (uint64_t)rows[d];
    R.fastmod_m = ~0ull / (uint64_t)ht_len[d] + 1ull;
    R.key_min = key_min[d];
    R.ht_len = ht_len[d];
    R.pred_kind = d < 2 ? SJ_PRED_IN : SJ_PRED_RANGE;
    R.pred_lo = INT32_MIN;  // date: d_year <= 1997 (0-lip.cu:187-190)
    R.pred_hi = 1997;
    R.payload_min = pmin[d];
    R.payload_span = span[d];
    R.grouped = 1;
    R.bf_mode = bpk ? kBfBlocked : kBfDirect;
    R.bf_k = bpk ? 2u : 1u;
    R.bf_bits_per_key = bpk;
    R.bf_max_log2 = bf_log2[d];
  }

  SjProbeGeom g;
  memset(&g, 0, sizeof(g));
  g.threads = 512;  // 15 consumer warps + 1 producer warp, 8 rows per lane
  g.chunk_rows = 15360;
  g.stages = 2;
  g.bf_smem_bytes = 40u * 1024u;
  rt.bf_smem_budget = g.bf_smem_bytes;
  g.group_smem_cap = 1024;
  g.q1_cap = 512;
  g.q2_cap = 128;  // room for a two-survivors-per-lane Q1 round (64) over a partial Q2
  g.reorder_period = 16;
  g.grid = (uint32_t)sms;
  g.smem_bytes = probe_smem_bytes(g);
  if (g.smem_bytes > (uint32_t)smem_optin)
    return na_fail(SJ_ERR_UNSUPPORTED, "probe needs %u bytes of shared memory per block; device %d allows %d",
                   g.smem_bytes, device, smem_optin);

  // ---- clear, upload the IN lists, build, probe, finalize, read back
  auto check = [&](cudaError_t ce, const char* what) -> sj_status {
    if (ce == cudaSuccess) return SJ_OK;
    cudaGetLastError();
    return na_fail(SJ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(ce));
  };
  if ((s = check(cudaMemsetAsync(base, 0, zero_bytes, st), "clearing scratch")) != SJ_OK) return s;
  for (int d = 0; d < 3; ++d)
    if ((s = check(cudaMemcpyAsync(base + inbm_off[d], in_bitmaps[d], sizeof(in_bitmaps[d]), cudaMemcpyHostToDevice,
                                   st),
                   "uploading IN lists")) != SJ_OK)
      return s;
  const int64_t max_rows = std::max(std::max(s_len, c_len), d_len);
  uint32_t bx = (uint32_t)std::min<int64_t>((max_rows + 255) / 256, (int64_t)sms * 8);
  dim3 grid(std::max(1u, bx), 3);
  sj_dim_scan<<<grid, 256, 0, st>>>(rt);
  if ((s = check(cudaGetLastError(), "dimension scan")) != SJ_OK) return s;
  sj_dim_insert<<<grid, 256, 4 * ((250 + 31) / 32), st>>>(rt);
  if ((s = check(cudaGetLastError(), "dimension insert")) != SJ_OK) return s;
  if (lo_len > 0 && (s = check(launch_probe(rt, g, 8, st, L2Window{}, false), "probe")) != SJ_OK) return s;
  if ((s = check(launch_finalize(rt, (uint32_t)groups, st, false), "finalize")) != SJ_OK) return s;
  SjDesc desc;
  if ((s = check(cudaMemcpyAsync(&desc, rt.desc, sizeof(desc), cudaMemcpyDeviceToHost, st), "reading status")) != SJ_OK)
    return s;
  if ((s = check(cudaStreamSynchronize(st), "synchronize")) != SJ_OK) return s;
  if (desc.error_flags & kErrWaitTimeout) return na_fail(SJ_ERR_TIMEOUT, "probe kernel: bounded wait expired");
  if (desc.error_flags & kErrPayloadDomain)
    return na_fail(SJ_ERR_INVALID_ARGUMENT, "a grouped payload lies outside [payload_min, payload_max]");
  if (desc.error_flags) return na_fail(SJ_ERR_CUDA, "device error flags 0x%x", desc.error_flags);
  *n_out = desc.groups_out;
  if ((int64_t)desc.groups_out > cap || (desc.groups_out && !out))
    return na_fail(SJ_ERR_CAPACITY, "need %u result rows", desc.groups_out);
  if (desc.groups_out) {
    if ((s = check(cudaMemcpyAsync(out, rt.rows_out, sizeof(sj_group_row) * desc.groups_out, cudaMemcpyDeviceToHost,
                                   st),
                   "reading groups")) != SJ_OK)
      return s;
    if ((s = check(cudaStreamSynchronize(st), "synchronize")) != SJ_OK) return s;
    std::sort(out, out + desc.groups_out, [](const sj_group_row& a, const sj_group_row& b) {
      for (int d = 0; d < SJ_MAX_DIMS; ++d)
        if (a.attr[d] != b.attr[d]) return a.attr[d] < b.attr[d];
      return false;
    });
  }
  return SJ_OK;
}
