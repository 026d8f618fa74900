// ref_runner.cu -- TEST INFRASTRUCTURE: a main() around one of the reference's
// own SSB Q3.3 drivers, compiled unmodified from its source tree by build_ref.py
// into oracle/_ref/.  It feeds the driver the seeded synthetic columns (the same
// generator the engine's tests use) instead of dbgen files, then
//   1. calls the driver's own runQuery() (src/ssb-jo/q33/<o>-<lip|naive>.cu) --
//      which prints "Result:" lines and returns its time_query (alloc + memsets +
//      builds + probe, src/ssb-jo/q33/0-lip.cu:216-278) -- for --t trials;
//   2. times the driver's probe<128,4> kernel alone (its builds done once) with
//      CUDA events over --probe_t launches.
// Output: the driver's own text plus one JSON line per measurement.
#define main crystal_reference_driver_main
#include REF_DRIVER
#undef main

#include <thread>
#include <vector>

#include "../crystal-opt_b200/csrc/sj_datagen.h"

static int* ref_gen_device(long long n, unsigned long long seed, int col, int kind, int lo, int hi) {
  int* h = new int[n > 0 ? n : 1];
  const uint64_t key = sj_stream_key(seed, (uint32_t)col);
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if (nt > 64) nt = 64;
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; ++t)
    pool.emplace_back([=]() {
      for (long long i = n * t / nt; i < n * (t + 1) / nt; ++i) h[i] = sj_gen_value(key, kind, lo, hi, (uint64_t)i);
    });
  for (auto& th : pool) th.join();
  int* d = loadToGPU<int>(h, (int)n, g_allocator);
  delete[] h;
  return d;
}

int main(int argc, char** argv) {
  CommandLineArgs args(argc, argv);
  unsigned long long seed = 1;
  int n = 6000000, c_len = 30000, s_len = 2000, trials = 1, probe_trials = 0;
  args.GetCmdLineArgument("seed", seed);
  args.GetCmdLineArgument("n", n);
  args.GetCmdLineArgument("c", c_len);
  args.GetCmdLineArgument("s", s_len);
  args.GetCmdLineArgument("t", trials);
  args.GetCmdLineArgument("probe_t", probe_trials);
  CubDebugExit(args.DeviceInit());
  const int d_len = SJ_DATE_DAYS;

  int* lo_orderdate = ref_gen_device(n, seed, SJ_COL_FK_DATE, SJ_GEN_DATEKEY, 0, 0);
  int* lo_custkey = ref_gen_device(n, seed, SJ_COL_FK_CUST, SJ_GEN_UNIFORM, 1, c_len);
  int* lo_suppkey = ref_gen_device(n, seed, SJ_COL_FK_SUPP, SJ_GEN_UNIFORM, 1, s_len);
  int* lo_revenue = ref_gen_device(n, seed, SJ_COL_REVENUE, SJ_GEN_UNIFORM, 1, 10000000);
  int* d_datekey = ref_gen_device(d_len, seed, 0, SJ_GEN_DATE_SEQ, 0, 0);
  int* d_year = ref_gen_device(d_len, seed, 0, SJ_GEN_DATE_YEAR, 0, 0);
  int* s_suppkey = ref_gen_device(s_len, seed, 0, SJ_GEN_SEQ, 1, 0);
  int* s_city = ref_gen_device(s_len, seed, SJ_COL_SUPP_CITY, SJ_GEN_UNIFORM, 0, 249);
  int* c_custkey = ref_gen_device(c_len, seed, 0, SJ_GEN_SEQ, 1, 0);
  int* c_city = ref_gen_device(c_len, seed, SJ_COL_CUST_CITY, SJ_GEN_UNIFORM, 0, 249);
  CubDebugExit(cudaDeviceSynchronize());

  for (int t = 0; t < trials; ++t) {
    float tq = runQuery(lo_orderdate, lo_custkey, lo_suppkey, lo_revenue, n, d_datekey, d_year, d_len, s_suppkey,
                        s_city, s_len, c_custkey, c_city, c_len, g_allocator);
    printf("{\"query\":33,\"time_query\":%.6f}\n", tq);
    fflush(stdout);
  }

  if (probe_trials > 0) {
    // The driver's own build + probe kernels with its own launch shapes
    // (src/ssb-jo/q33/0-lip.cu:244-274); builds once, probe timed alone.
    int *ht_d, *ht_c, *ht_s, *res;
    const int d_val_len = 19981230 - 19920101 + 1;
    CubDebugExit(cudaMalloc(&ht_d, 2 * d_val_len * sizeof(int)));
    CubDebugExit(cudaMalloc(&ht_s, 2 * s_len * sizeof(int)));
    CubDebugExit(cudaMalloc(&ht_c, 2 * c_len * sizeof(int)));
    CubDebugExit(cudaMemset(ht_d, 0, 2 * d_val_len * sizeof(int)));
    CubDebugExit(cudaMemset(ht_s, 0, 2 * s_len * sizeof(int)));
    CubDebugExit(cudaMemset(ht_c, 0, 2 * c_len * sizeof(int)));
    const int res_size = (1998 - 1992 + 1) * 250 * 250;
    CubDebugExit(cudaMalloc(&res, 4 * res_size * sizeof(int)));
    const int tile = 128 * 4;
#if REF_LIP
    uint32_t *bf_s, *bf_c, *bf_d;
    const int bf_s_size = (int)(roundUpToPowerOfTwo((uint32_t)s_len) / 32);
    const int bf_c_size = (int)(roundUpToPowerOfTwo((uint32_t)c_len) / 32);
    const int bf_d_size = (int)(roundUpToPowerOfTwo((uint32_t)d_val_len) / 32);
    CubDebugExit(cudaMalloc(&bf_s, bf_s_size * sizeof(uint32_t)));
    CubDebugExit(cudaMalloc(&bf_c, bf_c_size * sizeof(uint32_t)));
    CubDebugExit(cudaMalloc(&bf_d, bf_d_size * sizeof(uint32_t)));
    CubDebugExit(cudaMemset(bf_s, 0, bf_s_size * sizeof(uint32_t)));
    CubDebugExit(cudaMemset(bf_c, 0, bf_c_size * sizeof(uint32_t)));
    CubDebugExit(cudaMemset(bf_d, 0, bf_d_size * sizeof(uint32_t)));
    build_hashtable_s<128, 4><<<(s_len + tile - 1) / tile, 128>>>(s_suppkey, s_city, s_len, ht_s, s_len, bf_s,
                                                                   bf_s_size);
    build_hashtable_c<128, 4><<<(c_len + tile - 1) / tile, 128>>>(c_custkey, c_city, c_len, ht_c, c_len, bf_c,
                                                                   bf_c_size);
    build_hashtable_d<128, 4><<<(d_len + tile - 1) / tile, 128>>>(d_datekey, d_year, d_len, ht_d, d_val_len,
                                                                   19920101, bf_d, bf_d_size);
#else
    build_hashtable_s<128, 4><<<(s_len + tile - 1) / tile, 128>>>(s_suppkey, s_city, s_len, ht_s, s_len);
    build_hashtable_c<128, 4><<<(c_len + tile - 1) / tile, 128>>>(c_custkey, c_city, c_len, ht_c, c_len);
    build_hashtable_d<128, 4><<<(d_len + tile - 1) / tile, 128>>>(d_datekey, d_year, d_len, ht_d, d_val_len,
                                                                   19920101);
#endif
    CubDebugExit(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int t = 0; t < probe_trials; ++t) {
      CubDebugExit(cudaMemset(res, 0, 4 * res_size * sizeof(int)));
      cudaEventRecord(e0, 0);
#if REF_LIP
      probe<128, 4><<<(n + tile - 1) / tile, 128>>>(lo_orderdate, lo_custkey, lo_suppkey, lo_revenue, n, ht_s, s_len,
                                                    ht_c, c_len, ht_d, d_val_len, bf_s, bf_s_size, bf_c, bf_c_size,
                                                    bf_d, bf_d_size, res);
#else
      probe<128, 4><<<(n + tile - 1) / tile, 128>>>(lo_orderdate, lo_custkey, lo_suppkey, lo_revenue, n, ht_s, s_len,
                                                    ht_c, c_len, ht_d, d_val_len, res);
#endif
      cudaEventRecord(e1, 0);
      CubDebugExit(cudaEventSynchronize(e1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      printf("{\"probe_ms\":%.6f}\n", ms);
    }
    fflush(stdout);
  }
  return 0;
}
