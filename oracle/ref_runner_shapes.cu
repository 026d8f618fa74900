// ref_runner_shapes.cu -- TEST INFRASTRUCTURE: a main() around one of the
// reference's own SSB drivers other than Q3.3: src/ssb-jo/q{21,22,23,31,32,34,41}/0-lip.cu,
// src/ssb-jo/q42/0-naive.cu and src/ssb-jo/q43/q43.cu, compiled unmodified from
// its source tree by build_ref.py into oracle/_ref/.  It feeds the driver the
// seeded synthetic columns the engine's tests use (SSB's nested codes derived as
// nation = city / 10, region = city / 50, category = brand / 40,
// mfgr = brand / 200, d_yearmonthnum = datekey / 100) and calls the driver's
// own runQuery(), which prints one line per group, --t times (each followed by a
// {"query":Q,"time_query":ms} line: the driver's own timing of allocations,
// memsets, builds and probe).  REF_QUERY selects the driver.
#define main crystal_reference_driver_main
#include REF_DRIVER
#undef main

#include <thread>
#include <vector>

#include "../crystal-opt_b200/csrc/sj_datagen.h"

static std::vector<int> ref_gen_host(long long n, unsigned long long seed, int col, int kind, int lo, int hi) {
  std::vector<int> h((size_t)(n > 0 ? n : 1));
  const uint64_t key = sj_stream_key(seed, (uint32_t)col);
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if (nt > 64) nt = 64;
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; ++t)
    pool.emplace_back([&, t]() {
      for (long long i = n * t / nt; i < n * (t + 1) / nt; ++i) h[i] = sj_gen_value(key, kind, lo, hi, (uint64_t)i);
    });
  for (auto& th : pool) th.join();
  return h;
}

static std::vector<int> div_by(const std::vector<int>& v, int d) {
  std::vector<int> out(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = v[i] / d;
  return out;
}

static int* to_gpu(std::vector<int>& h, long long n) { return loadToGPU<int>(h.data(), (int)n, g_allocator); }

int main(int argc, char** argv) {
  CommandLineArgs args(argc, argv);
  unsigned long long seed = 1;
  int n = 6000000, c_len = 30000, s_len = 2000, p_len = 200000, trials = 1;
  args.GetCmdLineArgument("seed", seed);
  args.GetCmdLineArgument("t", trials);
  args.GetCmdLineArgument("n", n);
  args.GetCmdLineArgument("c", c_len);
  args.GetCmdLineArgument("s", s_len);
  args.GetCmdLineArgument("p", p_len);
  CubDebugExit(args.DeviceInit());
  const int d_len = SJ_DATE_DAYS;

  auto h_lo_orderdate = ref_gen_host(n, seed, SJ_COL_FK_DATE, SJ_GEN_DATEKEY, 0, 0);
  auto h_lo_custkey = ref_gen_host(n, seed, SJ_COL_FK_CUST, SJ_GEN_UNIFORM, 1, c_len);
  auto h_lo_suppkey = ref_gen_host(n, seed, SJ_COL_FK_SUPP, SJ_GEN_UNIFORM, 1, s_len);
  auto h_lo_partkey = ref_gen_host(n, seed, SJ_COL_FK_PART, SJ_GEN_UNIFORM, 1, p_len);
  auto h_lo_revenue = ref_gen_host(n, seed, SJ_COL_REVENUE, SJ_GEN_UNIFORM, 1, 10000000);
  auto h_lo_supplycost = ref_gen_host(n, seed, SJ_COL_SUPPLYCOST, SJ_GEN_UNIFORM, 1, 100000);
  auto h_d_datekey = ref_gen_host(d_len, seed, 0, SJ_GEN_DATE_SEQ, 0, 0);
  auto h_d_year = ref_gen_host(d_len, seed, 0, SJ_GEN_DATE_YEAR, 0, 0);
  auto h_s_suppkey = ref_gen_host(s_len, seed, 0, SJ_GEN_SEQ, 1, 0);
  auto h_s_city = ref_gen_host(s_len, seed, SJ_COL_SUPP_CITY, SJ_GEN_UNIFORM, 0, 249);
  auto h_c_custkey = ref_gen_host(c_len, seed, 0, SJ_GEN_SEQ, 1, 0);
  auto h_c_city = ref_gen_host(c_len, seed, SJ_COL_CUST_CITY, SJ_GEN_UNIFORM, 0, 249);
  auto h_p_partkey = ref_gen_host(p_len, seed, 0, SJ_GEN_SEQ, 1, 0);
  auto h_p_brand1 = ref_gen_host(p_len, seed, SJ_COL_PART_BRAND, SJ_GEN_UNIFORM, 0, 999);
  auto h_s_nation = div_by(h_s_city, 10), h_s_region = div_by(h_s_city, 50);
  auto h_c_nation = div_by(h_c_city, 10), h_c_region = div_by(h_c_city, 50);
  auto h_p_category = div_by(h_p_brand1, 40), h_p_mfgr = div_by(h_p_brand1, 200);
  auto h_d_yearmonthnum = div_by(h_d_datekey, 100);

  int* lo_orderdate = to_gpu(h_lo_orderdate, n);
  int* lo_suppkey = to_gpu(h_lo_suppkey, n);
  int* lo_revenue = to_gpu(h_lo_revenue, n);
  int* d_datekey = to_gpu(h_d_datekey, d_len);
  int* d_year = to_gpu(h_d_year, d_len);
  int* s_suppkey = to_gpu(h_s_suppkey, s_len);
  int* s_region = to_gpu(h_s_region, s_len);
  printf("Result:\n");
#if REF_QUERY == 21
  int* lo_partkey = to_gpu(h_lo_partkey, n);
  int* p_partkey = to_gpu(h_p_partkey, p_len);
  int* p_brand1 = to_gpu(h_p_brand1, p_len);
  int* p_category = to_gpu(h_p_category, p_len);
  CubDebugExit(cudaDeviceSynchronize());
  fflush(stdout);
  for (int t = 0; t < trials; ++t) {
    const float tq = runQuery(lo_orderdate, lo_partkey, lo_suppkey, lo_revenue, n, p_partkey, p_brand1, p_category, p_len, d_datekey,
           d_year, d_len, s_suppkey, s_region, s_len, g_allocator);
    printf("{\"query\":%d,\"time_query\":%.6f}\n", REF_QUERY, tq);
    fflush(stdout);
  }
#elif REF_QUERY == 22 || REF_QUERY == 23
  int* lo_partkey = to_gpu(h_lo_partkey, n);
  int* p_partkey = to_gpu(h_p_partkey, p_len);
  int* p_brand1 = to_gpu(h_p_brand1, p_len);
  CubDebugExit(cudaDeviceSynchronize());
  fflush(stdout);
  for (int t = 0; t < trials; ++t) {
    const float tq = runQuery(lo_orderdate, lo_partkey, lo_suppkey, lo_revenue, n, p_partkey, p_brand1, p_len, d_datekey, d_year, d_len,
           s_suppkey, s_region, s_len, g_allocator);
    printf("{\"query\":%d,\"time_query\":%.6f}\n", REF_QUERY, tq);
    fflush(stdout);
  }
#elif REF_QUERY == 32
  int* lo_custkey = to_gpu(h_lo_custkey, n);
  int* s_nation = to_gpu(h_s_nation, s_len);
  int* s_city = to_gpu(h_s_city, s_len);
  int* c_custkey = to_gpu(h_c_custkey, c_len);
  int* c_nation = to_gpu(h_c_nation, c_len);
  int* c_city = to_gpu(h_c_city, c_len);
  CubDebugExit(cudaDeviceSynchronize());
  fflush(stdout);
  for (int t = 0; t < trials; ++t) {
    const float tq = runQuery(lo_orderdate, lo_custkey, lo_suppkey, lo_revenue, n, d_datekey, d_year, d_len, s_suppkey, s_nation,
           s_city, s_len, c_custkey, c_nation, c_city, c_len, g_allocator);
    printf("{\"query\":%d,\"time_query\":%.6f}\n", REF_QUERY, tq);
    fflush(stdout);
  }
#elif REF_QUERY == 34
  int* lo_custkey = to_gpu(h_lo_custkey, n);
  int* d_yearmonthnum = to_gpu(h_d_yearmonthnum, d_len);
  int* s_city = to_gpu(h_s_city, s_len);
  int* c_custkey = to_gpu(h_c_custkey, c_len);
  int* c_city = to_gpu(h_c_city, c_len);
  CubDebugExit(cudaDeviceSynchronize());
  fflush(stdout);
  for (int t = 0; t < trials; ++t) {
    const float tq = runQuery(lo_orderdate, lo_custkey, lo_suppkey, lo_revenue, n, d_datekey, d_year, d_yearmonthnum, d_len,
           s_suppkey, s_city, s_len, c_custkey, c_city, c_len, g_allocator);
    printf("{\"query\":%d,\"time_query\":%.6f}\n", REF_QUERY, tq);
    fflush(stdout);
  }
#elif REF_QUERY == 31
  int* lo_custkey = to_gpu(h_lo_custkey, n);
  int* s_nation = to_gpu(h_s_nation, s_len);
  int* c_custkey = to_gpu(h_c_custkey, c_len);
  int* c_region = to_gpu(h_c_region, c_len);
  int* c_nation = to_gpu(h_c_nation, c_len);
  CubDebugExit(cudaDeviceSynchronize());
  fflush(stdout);
  for (int t = 0; t < trials; ++t) {
    const float tq = runQuery(lo_orderdate, lo_custkey, lo_suppkey, lo_revenue, n, d_datekey, d_year, d_len, s_suppkey, s_region,
           s_nation, s_len, c_custkey, c_region, c_nation, c_len, g_allocator);
    printf("{\"query\":%d,\"time_query\":%.6f}\n", REF_QUERY, tq);
    fflush(stdout);
  }
#elif REF_QUERY == 41
  int* lo_custkey = to_gpu(h_lo_custkey, n);
  int* lo_partkey = to_gpu(h_lo_partkey, n);
  int* lo_supplycost = to_gpu(h_lo_supplycost, n);
  int* p_partkey = to_gpu(h_p_partkey, p_len);
  int* p_mfgr = to_gpu(h_p_mfgr, p_len);
  int* c_custkey = to_gpu(h_c_custkey, c_len);
  int* c_region = to_gpu(h_c_region, c_len);
  int* c_nation = to_gpu(h_c_nation, c_len);
  CubDebugExit(cudaDeviceSynchronize());
  fflush(stdout);
  for (int t = 0; t < trials; ++t) {
    const float tq = runQuery(lo_orderdate, lo_custkey, lo_partkey, lo_suppkey, lo_revenue, lo_supplycost, n, d_datekey, d_year, d_len,
           p_partkey, p_mfgr, p_len, s_suppkey, s_region, s_len, c_custkey, c_region, c_nation, c_len, g_allocator);
    printf("{\"query\":%d,\"time_query\":%.6f}\n", REF_QUERY, tq);
    fflush(stdout);
  }
#elif REF_QUERY == 42
  int* lo_custkey = to_gpu(h_lo_custkey, n);
  int* lo_partkey = to_gpu(h_lo_partkey, n);
  int* lo_supplycost = to_gpu(h_lo_supplycost, n);
  int* p_partkey = to_gpu(h_p_partkey, p_len);
  int* p_mfgr = to_gpu(h_p_mfgr, p_len);
  int* p_category = to_gpu(h_p_category, p_len);
  int* s_nation = to_gpu(h_s_nation, s_len);
  int* c_custkey = to_gpu(h_c_custkey, c_len);
  int* c_region = to_gpu(h_c_region, c_len);
  CubDebugExit(cudaDeviceSynchronize());
  fflush(stdout);
  for (int t = 0; t < trials; ++t) {
    const float tq = runQuery(lo_orderdate, lo_custkey, lo_partkey, lo_suppkey, lo_revenue, lo_supplycost, n, d_datekey, d_year, d_len,
           p_partkey, p_mfgr, p_category, p_len, s_suppkey, s_region, s_nation, s_len, c_custkey, c_region, c_len,
           g_allocator);
    printf("{\"query\":%d,\"time_query\":%.6f}\n", REF_QUERY, tq);
    fflush(stdout);
  }
#elif REF_QUERY == 43
  int* lo_custkey = to_gpu(h_lo_custkey, n);
  int* lo_partkey = to_gpu(h_lo_partkey, n);
  int* lo_supplycost = to_gpu(h_lo_supplycost, n);
  int* p_partkey = to_gpu(h_p_partkey, p_len);
  int* p_category = to_gpu(h_p_category, p_len);
  int* p_brand1 = to_gpu(h_p_brand1, p_len);
  int* s_nation = to_gpu(h_s_nation, s_len);
  int* s_city = to_gpu(h_s_city, s_len);
  int* c_custkey = to_gpu(h_c_custkey, c_len);
  int* c_region = to_gpu(h_c_region, c_len);
  CubDebugExit(cudaDeviceSynchronize());
  fflush(stdout);
  for (int t = 0; t < trials; ++t) {
    const float tq = runQuery(lo_orderdate, lo_custkey, lo_partkey, lo_suppkey, lo_revenue, lo_supplycost, n, d_datekey, d_year, d_len,
           p_partkey, p_category, p_brand1, p_len, s_suppkey, s_nation, s_city, s_len, c_custkey, c_region, c_len,
           g_allocator);
    printf("{\"query\":%d,\"time_query\":%.6f}\n", REF_QUERY, tq);
    fflush(stdout);
  }
#else
#error "REF_QUERY must be 21, 22, 23, 31, 32, 34, 41, 42 or 43"
#endif
  fflush(stdout);
  return 0;
}
