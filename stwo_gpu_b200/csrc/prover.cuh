// The prover's entry points shared by the C API (prover.cu) and the proof server
// (server.cu).
#pragma once
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace stwo {

// A server worker's retained proof slab and the CUDA graph of the proof's launch
// sequence on it, for proving the same job shape again: the first proof of a shape
// keeps its slab here, the second (same shape, same twiddle tree, same device) reuses
// it and captures its launch sequence, later ones replay the graph.
struct ProveCache {
    bool valid = false;
    uint32_t key[5] = {};  // log_n_rows, n_columns, log_blowup, n_queries, pow_bits
    uint64_t tunables_gen = 0;  // tunables_generation() when the slab and graph were made
    const uint32_t *tw = nullptr, *itw = nullptr;
    uint64_t tsz = 0;
    int device = -1;
    uint8_t *slab = nullptr;
    uint64_t cap = 0;
    cudaGraphExec_t exec = nullptr;
    bool no_graph = false;  // the launch sequence did not capture: run it directly
    uint64_t launches = 0;  // kernel launches inside the graph
    uint64_t replays = 0;   // graph replays over the cache's life
};

// Frees the slab (stream-ordered on st) and the graph, and empties the cache (the
// replay count runs on).
void prove_cache_release(ProveCache *c, cudaStream_t st);

// One proof. cache: optional (server workers pass theirs).
int wide_fib_prove(const stwo_wide_fib_job *job, const uint32_t *a0, const uint32_t *a1, const uint32_t *tw,
                   const uint32_t *itw, uint64_t tree_size, std::vector<uint8_t> &proof, stwo_prove_stats *stats,
                   cudaStream_t st, ProveCache *cache = nullptr);
uint64_t wide_fib_job_device_bytes(const stwo_wide_fib_job *job, bool own_twiddles);
// n_jobs proofs of one shape in one launch sequence (the caller's twiddle tree):
// proofs[k], job_rc[k] receive job k's bytes and status.
int wide_fib_prove_batch(const stwo_wide_fib_job *job, uint32_t n_jobs, const uint32_t *const *a0,
                         const uint32_t *const *a1, const uint32_t *tw, const uint32_t *itw, uint64_t tree_size,
                         std::vector<std::vector<uint8_t>> &proofs, int *job_rc, stwo_prove_stats *stats,
                         cudaStream_t st);

}  // namespace stwo
