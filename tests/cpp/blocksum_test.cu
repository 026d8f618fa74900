// blocksum_test.cu -- GPU check of the drop-in BlockSum (crystal/reduce.cuh;
// the reference's is crystal/reduce.cuh:25-75).  Every block loads one striped
// tile with BlockLoad (the last tile partial), sums it with both BlockSum
// overloads -- the register-array form and the per-thread scalar form, the
// latter as src/ops/bloom_join.cu:98-110 calls it for long long -- and thread 0
// writes the block total.  The host sums the same tiles and compares.
//
// Prints one line per case, "ok <type> <threads> <items> <tiles> <n>", or
// "FAIL ..." and exits 1 on the first mismatch.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "crystal/crystal.cuh"

template <typename T, int BT, int IPT>
__global__ void tile_sums(const T* in, int n, T* out_items, T* out_scalar) {
  __shared__ T buf[32];
  const int tile = BT * IPT;
  const int off = blockIdx.x * tile;
  const int num = (n - off) < tile ? (n - off) : tile;
  T items[IPT];
#pragma unroll
  for (int i = 0; i < IPT; ++i) items[i] = 0;
  BlockLoad<T, BT, IPT>(const_cast<T*>(in) + off, items, num);  // unguarded when num == tile
  const T a = BlockSum<T, BT, IPT>(items, buf);
  if (threadIdx.x == 0) out_items[blockIdx.x] = a;
  T s = 0;
#pragma unroll
  for (int i = 0; i < IPT; ++i)
    if ((int)threadIdx.x + BT * i < num) s += items[i];
  const T b = BlockSum<T, BT, IPT>(s, buf);
  if (threadIdx.x == 0) out_scalar[blockIdx.x] = b;
}

static uint64_t g_state = 0x243F6A8885A308D3ull;
static uint64_t next_u64() {  // SplitMix64 (Steele, Lea, Flood 2014)
  uint64_t z = (g_state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <typename T>
T draw();
template <>
int draw<int>() { return (int)(next_u64() % 2000001ull) - 1000000; }
template <>
unsigned draw<unsigned>() { return (unsigned)(next_u64() % 2000001ull); }
template <>
long long draw<long long>() { return (long long)(next_u64() % 2000000000001ull) - 1000000000000ll; }

template <typename T>
const char* tname();
template <>
const char* tname<int>() { return "int"; }
template <>
const char* tname<unsigned>() { return "unsigned"; }
template <>
const char* tname<long long>() { return "long_long"; }

#define CK(x)                                                                  \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess) {                                                   \
      printf("FAIL cuda %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return false;                                                            \
    }                                                                          \
  } while (0)

template <typename T, int BT, int IPT>
bool run_case(int n) {
  const int tile = BT * IPT;
  const int tiles = (n + tile - 1) / tile;
  std::vector<T> h(n);
  for (auto& v : h) v = draw<T>();
  T *d_in = nullptr, *d_a = nullptr, *d_b = nullptr;
  CK(cudaMalloc(&d_in, sizeof(T) * (size_t)n));
  CK(cudaMalloc(&d_a, sizeof(T) * (size_t)tiles));
  CK(cudaMalloc(&d_b, sizeof(T) * (size_t)tiles));
  CK(cudaMemcpy(d_in, h.data(), sizeof(T) * (size_t)n, cudaMemcpyHostToDevice));
  tile_sums<T, BT, IPT><<<tiles, BT>>>(d_in, n, d_a, d_b);
  CK(cudaGetLastError());
  std::vector<T> a(tiles), b(tiles);
  CK(cudaMemcpy(a.data(), d_a, sizeof(T) * (size_t)tiles, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(b.data(), d_b, sizeof(T) * (size_t)tiles, cudaMemcpyDeviceToHost));
  cudaFree(d_in);
  cudaFree(d_a);
  cudaFree(d_b);
  for (int t = 0; t < tiles; ++t) {
    T want = 0;
    for (int i = t * tile; i < n && i < (t + 1) * tile; ++i) want += h[i];
    if (a[t] != want || b[t] != want) {
      printf("FAIL %s %d %d tile %d of %d: items %lld scalar %lld host %lld\n", tname<T>(), BT, IPT, t, tiles,
             (long long)a[t], (long long)b[t], (long long)want);
      return false;
    }
  }
  printf("ok %s %d %d %d %d\n", tname<T>(), BT, IPT, tiles, n);
  return true;
}

int main() {
  bool ok = true;
  // the reference drivers' geometry (128 x 4), a full grid and a ragged last tile
  ok = ok && run_case<int, 128, 4>(512 * 64);
  ok = ok && run_case<int, 128, 4>(512 * 37 + 101);
  ok = ok && run_case<unsigned, 128, 4>(512 * 37 + 1);
  ok = ok && run_case<long long, 128, 4>(512 * 37 + 511);
  // one warp, wider blocks, one item per thread
  ok = ok && run_case<int, 32, 4>(128 * 9 + 7);
  ok = ok && run_case<long long, 256, 2>(512 * 11 + 3);
  ok = ok && run_case<unsigned, 1024, 1>(1024 * 5 + 1000);
  ok = ok && run_case<long long, 1024, 4>(4096 * 3 + 17);
  // a single partial tile smaller than one warp
  ok = ok && run_case<int, 128, 4>(5);
  return ok ? 0 : 1;
}
