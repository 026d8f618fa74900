// sj_build.cu -- stand-alone dimension-build kernels: predicate evaluation,
// payload dictionary, perfect-hash-table insert and Bloom-filter insert.
//
// Replaces the reference's build_hashtable_{s,c,d} kernels
// (src/ssb-jo/q33/0-lip.cu:114-203).  Two launches per query, each covering every
// dimension (blockIdx.y = dim):
//   sj_dim_scan   clears the hash tables and filters, lists the qualifying rows
//                 (their count sizes the filter) and marks their payloads in a
//                 bitmap over the payload domain (the group-key dictionary);
//   sj_dim_insert sizes the filter from the count (bits per inserted key), ranks
//                 payloads into dense group codes, and inserts the listed rows into
//                 the PHT ([key, code] slots, the reference's 2 x int32 layout) and
//                 the filter.
// Everything the probe needs (filter geometry, code counts, group strides, the
// starting LIP order) is written to the query descriptor on the device: no host
// round trip, so a whole query can be captured in a CUDA graph.
#include "sj_build.cuh"

namespace sj {

// Clears the descriptor and payload bitmaps a build starts from (16-byte
// multiple); the scan kernel, launched as its programmatic dependent, clears the
// hash tables meanwhile and waits for this grid before its first write there.
__global__ void __launch_bounds__(256) sj_clear_head(uint4* __restrict__ head, uint64_t n16) {
  pdl_launch_dependents();
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x)
    head[i] = make_uint4(0u, 0u, 0u, 0u);
}

__global__ void __launch_bounds__(256) sj_dim_scan(const __grid_constant__ SjPlanRt P) {
  pdl_launch_dependents();  // sj_dim_insert may be scheduled; it waits for this grid
  // clear the hash tables and filters sj_dim_insert fills (every block of the grid)
  if (P.zero_tables_bytes) {
    uint4* z = reinterpret_cast<uint4*>(P.zero_tables);
    const uint64_t n = P.zero_tables_bytes / 16u;
    const uint64_t nt = (uint64_t)gridDim.x * gridDim.y * blockDim.x;
    for (uint64_t i = ((uint64_t)blockIdx.y * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += nt)
      z[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  pdl_wait();  // launched after sj_clear_head: the descriptor and payload bitmaps are clear
  const uint32_t d = blockIdx.y;
  if (d >= P.n_dims) return;
  SjDesc* desc = P.desc;
  dim_scan_rows(P, d, blockIdx.x, gridDim.x, &desc->error_flags, &desc->dim[d].n_inserted);
}

__global__ void __launch_bounds__(256) sj_dim_insert(const __grid_constant__ SjPlanRt P) {
  pdl_launch_dependents();  // the probe may be scheduled; it waits for this grid
  pdl_wait();               // sj_dim_scan's counts and payload bitmaps are complete
  extern __shared__ uint32_t prefix[];  // payload-bitmap prefix popcounts
  __shared__ uint32_t s_total;
  const uint32_t d = blockIdx.y;
  if (d >= P.n_dims) return;
  const SjDimRt& D = P.dim[d];
  SjDesc* desc = P.desc;

  const uint32_t n_ins = desc->dim[d].n_inserted;
  uint32_t log2;
  const uint32_t mode = bf_effective(D.bf_mode, D.bf_max_log2, D.bf_bits_per_key, n_ins, P.bf_smem_budget, &log2);
  const uint32_t pwords = D.grouped ? (D.payload_span + 31u) / 32u : 0u;
  if (D.grouped) {
    if (threadIdx.x < 32) warp_bitmap_prefix(D.payload_bitmap, pwords, prefix, &s_total, threadIdx.x);
    __syncthreads();
  }

  if (blockIdx.x == 0) {
    if (threadIdx.x == 0) {
      desc->dim[d].bf_log2 = log2;
      desc->dim[d].bf_mode = mode;
    }
    if (D.grouped) {
      write_dict(D, prefix, pwords);
      if (threadIdx.x == 0) desc->dim[d].n_codes = s_total;
    }
  }
  // the query-wide fields, by warp 0 of dimension 0's last block: the blocks at
  // the front of the grid take the listed rows, so this overlaps the inserts
  if (blockIdx.x == gridDim.x - 1) {
    if (d == 0 && threadIdx.x < 32) {
      const uint32_t lane = threadIdx.x;
      uint32_t n_codes[kMaxDims] = {0, 0, 0, 0}, stride[kMaxDims], ins[kMaxDims] = {0, 0, 0, 0};
#pragma unroll
      for (uint32_t e = 0; e < kMaxDims; ++e) {
        if (e >= P.n_dims) continue;
        ins[e] = desc->dim[e].n_inserted;
        if (!P.dim[e].grouped) continue;
        const uint32_t ew = (P.dim[e].payload_span + 31u) / 32u;
        uint32_t c = 0;
        for (uint32_t w = lane; w < ew; w += 32) c += __popc(P.dim[e].payload_bitmap[w]);
        n_codes[e] = __reduce_add_sync(0xffffffffu, c);
      }
      if (lane == 0) {
        desc->n_groups = group_strides(P, n_codes, stride);
        for (uint32_t e = 0; e < P.n_dims; ++e) desc->dim[e].group_stride = stride[e];
      }
      choose_start(P, ins, desc->start_order, desc->bf_smem_off, lane);
    }
  }
  dim_insert_rows(P, d, mode, log2, prefix, n_ins, blockIdx.x, gridDim.x);
}

}  // namespace sj
