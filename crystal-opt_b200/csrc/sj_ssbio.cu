// sj_ssbio.cu -- the reference's on-disk column layout (sj_ssb_* in include/starjoin.h).
//
// The reference keeps each SSB column in its own headerless file of native
// (little-endian) int32 values, named by table and by the column's position in
// that table's SSB column list: lo_custkey -> LINEORDER2, d_year -> DDATE4
// (src/ssb/ssb_utils.h:106-153 lookup(), :161-171 loadColumn()).  Host code only.
#include <cstdio>
#include <cstring>
#include <string>

#include "sj_cache.h"
#include "sj_internal.h"

using namespace sj;

namespace {

// SSB column order per table (the positions give the file suffix).
const char* const kLineorder[] = {"lo_orderkey",  "lo_linenumber",  "lo_custkey",       "lo_partkey",
                                  "lo_suppkey",   "lo_orderdate",   "lo_orderpriority", "lo_shippriority",
                                  "lo_quantity",  "lo_extendedprice", "lo_ordtotalprice", "lo_discount",
                                  "lo_revenue",   "lo_supplycost",  "lo_tax",           "lo_commitdate",
                                  "lo_shipmode"};
const char* const kPart[] = {"p_partkey", "p_name", "p_mfgr",  "p_category", "p_brand1",
                             "p_color",   "p_type", "p_size",  "p_container"};
const char* const kSupplier[] = {"s_suppkey", "s_name", "s_address", "s_city", "s_nation", "s_region", "s_phone"};
const char* const kCustomer[] = {"c_custkey", "c_name",   "c_address", "c_city",
                                 "c_nation",  "c_region", "c_phone",   "c_mktsegment"};
const char* const kDate[] = {"d_datekey",       "d_date",           "d_dayofweek",      "d_month",
                             "d_year",          "d_yearmonthnum",   "d_yearmonth",      "d_daynuminweek",
                             "d_daynuminmonth", "d_daynuminyear",   "d_sellingseason",  "d_lastdayinweekfl",
                             "d_lastdayinmonthfl", "d_holidayfl",   "d_weekdayfl"};

struct Table {
  const char* prefix;
  const char* const* cols;
  int n;
};

const Table kTables[] = {{"LINEORDER", kLineorder, 17}, {"PART", kPart, 9},      {"SUPPLIER", kSupplier, 7},
                         {"CUSTOMER", kCustomer, 8},    {"DDATE", kDate, 15}};

bool file_name(const char* col, std::string* out) {
  if (!col) return false;
  for (const Table& t : kTables)
    for (int i = 0; i < t.n; ++i)
      if (std::strcmp(col, t.cols[i]) == 0) {
        *out = std::string(t.prefix) + std::to_string(i);
        return true;
      }
  return false;
}

std::string join(const char* dir, const std::string& name) {
  std::string d = dir ? dir : "";
  if (!d.empty() && d.back() != '/') d += '/';
  return d + name;
}

}  // namespace

extern "C" sj_status sj_ssb_column_file(const char* column, char* out, int64_t cap) {
  std::string name;
  if (!file_name(column, &name)) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "not an SSB column: %s", column ? column : "(null)");
  if (!out || cap < (int64_t)name.size() + 1)
    return fail_fmt(SJ_ERR_CAPACITY, "file name %s needs %zu bytes", name.c_str(), name.size() + 1);
  std::memcpy(out, name.c_str(), name.size() + 1);
  return SJ_OK;
}

extern "C" sj_status sj_ssb_load_column(const char* dir, const char* column, int64_t n, int32_t* out) {
  std::string name;
  if (!file_name(column, &name)) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "not an SSB column: %s", column ? column : "(null)");
  if (n < 0 || (n > 0 && !out)) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "n=%lld, out=%p", (long long)n, (void*)out);
  const std::string path = join(dir, name);
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "cannot open %s", path.c_str());
  const size_t got = n ? std::fread(out, sizeof(int32_t), (size_t)n, f) : 0;
  std::fclose(f);
  if (got != (size_t)n)
    return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "%s holds %zu values, %lld asked", path.c_str(), got, (long long)n);
  return SJ_OK;
}

extern "C" sj_status sj_ssb_store_column(const char* dir, const char* column, int64_t n, const int32_t* data) {
  std::string name;
  if (!file_name(column, &name)) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "not an SSB column: %s", column ? column : "(null)");
  if (n < 0 || (n > 0 && !data)) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "n=%lld, data=%p", (long long)n, (const void*)data);
  const std::string path = join(dir, name);
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "cannot create %s", path.c_str());
  const size_t put = n ? std::fwrite(data, sizeof(int32_t), (size_t)n, f) : 0;
  const bool ok = std::fclose(f) == 0 && put == (size_t)n;
  return ok ? SJ_OK : fail_fmt(SJ_ERR_INVALID_ARGUMENT, "short write to %s", path.c_str());
}
