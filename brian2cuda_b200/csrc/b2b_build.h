// Host-callable connectivity build helpers (implemented in build.cu).
#pragma once
#include "b2b_internal.h"

namespace b2b {
// Keys (i - pre_lo)*nd + (delay - dmin) and input positions of one Synapses object;
// counts every key into d_counts[key_base + key].
cudaError_t member_keys(const int32_t* d_i, const int32_t* d_d, int64_t n, int32_t pre_lo,
                        int32_t nd, int32_t dmin, int64_t key_base, uint32_t* d_keys,
                        uint32_t* d_vals, int64_t* d_counts, cudaStream_t s);
// Exclusive scan of nkeys+1 counts in place; *max_count receives the largest count.
cudaError_t counts_to_offsets(int64_t* d_counts, int64_t nkeys, int64_t* max_count,
                              cudaStream_t s);
// Stable sort of one member by key, then scatter of targets/weights to their positions.
cudaError_t member_sort_scatter(uint32_t* d_keys, uint32_t* d_vals, int64_t n,
                                uint64_t max_key, const int64_t* d_off, int64_t key_base,
                                const int32_t* d_j, int64_t dst_offset, const void* d_w,
                                int dtype, int32_t* d_post, void* d_wout, int64_t* d_inv,
                                cudaStream_t s);
cudaError_t fill_value(void* d, int dtype, int64_t n, double v, cudaStream_t s);
// connect(p) with per-synapse uniform integer delays; arrays in (i, j) order.
// Rows i in [pre_lo, pre_hi) (keys use i as given); arrays in (i, j) order.
cudaError_t generate_random_ijd(int64_t pre_lo, int64_t pre_hi, int64_t n_post, double p,
                                int32_t dmin, int32_t dmax, uint64_t seed, int32_t** d_i,
                                int32_t** d_j, int32_t** d_d, int64_t* n_syn, cudaStream_t s);
// Post-sorted index of a projection's synapses (for on_post pathways).
cudaError_t build_post_index(const int32_t* d_post, int64_t n_syn, int64_t dst_lo,
                             int64_t n_dst, int64_t* d_post_off, int32_t* d_post_syn,
                             int64_t* max_count, cudaStream_t s);
cudaError_t gather_syn_var(const Proj& pr, int var, const int64_t* d_inv, int64_t pos_base,
                           int64_t n, int64_t key_lo, int64_t key_hi, int64_t src_offset,
                           int64_t dst_offset, const void* d_arr, int64_t stride,
                           double w_scalar, void* d_out, cudaStream_t s);
// Adds the out-degree (all delays) of source neurons [first, first + n) into d_out.
cudaError_t add_out_degree(const int64_t* d_off, int32_t nd, int64_t first, int64_t n,
                           int32_t* d_out, cudaStream_t s);
// STDP records from synapse order into post-grouped order (record r = synapse post_syn[r]) or
// back, d_in -> d_out (distinct buffers).
cudaError_t permute_stdp_records(const void* d_in, void* d_out, const int32_t* d_post_syn,
                                 int64_t n, int dtype, bool to_post, cudaStream_t s);
// rec_of[post_syn[r]] = r: the post-grouped record of each synapse position.
cudaError_t build_rec_of(const int32_t* d_post_syn, int64_t n, int32_t* d_rec_of,
                         cudaStream_t s);
// Interleaved STDP records {w, Apre = 0, Apost = 0, lastupdate = 0} from initial weights.
cudaError_t pack_stdp(const void* d_w, void* d_syn4, int dtype, int64_t n, cudaStream_t s);
}  // namespace b2b
