// stwo_autotune: measures the library's launch-parameter variants on the current
// device and keeps the fastest per size class (the Tunable table in common.cuh):
//
//   FFT elements per thread (2^5 or 2^6), separately for contiguous passes on domains
//   up to 2^20, contiguous passes on larger domains, and strided passes; measured on 8
//   columns interpolated at 2^18 / 2^22 and evaluated at blowup 4;
//   Merkle layers per launch (CTA of 128, 256 or 512 threads); measured on a tree of
//   64 columns x 2^19 leaves;
//   Merkle bottom-level nodes per thread (2^1 .. 2^5); measured on a tree of 4
//   columns x 2^20 leaves;
//   FFT radix split: the most layers a strided pass takes (10, 7 or 5: one strided
//   pass above the bottom pass, or two); measured like the elements per thread, at 2^22.
//
// Each candidate runs once to warm up, then three times; the least time wins. Every
// variant computes the same values, so tuning changes speed only. Device memory for
// the measurement comes from the library pool and is returned.
#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "common.cuh"

namespace stwo {

int fft_columns(const uint32_t *const *srcs, uint32_t *const *dsts, uint32_t n_cols, uint32_t N, uint32_t L,
                const uint32_t *tree, uint64_t tree_size, bool inv, cudaStream_t st);
int merkle_tree_dev_async(uint32_t max_log, const uint32_t *const *const *level_cols, const uint32_t *level_ncols,
                          uint32_t *const *layers, uint32_t *tickets, uint32_t n_tickets, uint32_t jobs, size_t js,
                          cudaStream_t st);
int butterfly_probe_async(uint32_t iters, uint32_t *sink, uint64_t sink_words, uint64_t *butterflies,
                          cudaStream_t st);

namespace {

// Ticket words for the Merkle tree kernel: more than any tree timed here needs.
constexpr uint32_t TICKETS = 1024;

struct Buffers {
    cudaStream_t st;
    std::vector<void *> ptrs;
    explicit Buffers(cudaStream_t s) : st(s) {}
    ~Buffers() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
    }
    uint32_t *get(size_t words) {
        void *p = nullptr;
        if (pool_alloc(&p, std::max<size_t>(words, 4) * 4, st) != STWO_OK) return nullptr;
        ptrs.push_back(p);
        return static_cast<uint32_t *>(p);
    }
};

__global__ void fill_kernel(uint32_t *p, uint64_t n, uint32_t seed) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = (i + 1) * 0x9E3779B97F4A7C15ull + seed;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        p[i] = (uint32_t)((z ^ (z >> 31)) % P);
    }
}

// Least time in ms of three runs of fn after one warm-up run.
template <class F>
int time_best(cudaStream_t st, F fn, float *best) {
    cudaEvent_t a, b;
    STWO_CUDA_TRY(cudaEventCreate(&a));
    STWO_CUDA_TRY(cudaEventCreate(&b));
    int rc = fn();
    *best = 1e30f;
    for (int r = 0; rc == STWO_OK && r < 3; r++) {
        cudaEventRecord(a, st);
        rc = fn();
        cudaEventRecord(b, st);
        if (rc == STWO_OK && cudaEventSynchronize(b) == cudaSuccess) {
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            *best = std::min(*best, ms);
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

}  // namespace
}  // namespace stwo

using namespace stwo;

extern "C" {

int stwo_set_tunable(const char *name, int value) {
    STWO_REQUIRE(name, STWO_ERR_INVALID_ARGUMENT, "null tunable name");
    const std::string n(name);
    if (n == "fft_ept_contig_small" || n == "fft_ept_contig_large" || n == "fft_ept_strided") {
        STWO_REQUIRE(value == 5 || value == 6, STWO_ERR_INVALID_ARGUMENT, "%s must be 5 or 6", name);
        set_tunable(n == "fft_ept_contig_small" ? TUNE_FFT_EPT_CONTIG_SMALL
                    : n == "fft_ept_contig_large" ? TUNE_FFT_EPT_CONTIG_LARGE : TUNE_FFT_EPT_STRIDED, value);
        return STWO_OK;
    }
    if (n == "merkle_sub_threads") {
        STWO_REQUIRE(value == 128 || value == 256 || value == 512, STWO_ERR_INVALID_ARGUMENT,
                     "merkle_sub_threads must be 128, 256 or 512");
        set_tunable(TUNE_MERKLE_SUB_THREADS, value);
        return STWO_OK;
    }
    if (n == "merkle_sub_spread") {
        STWO_REQUIRE(value >= 0 && value <= 5, STWO_ERR_INVALID_ARGUMENT, "merkle_sub_spread must be 0..5");
        set_tunable(TUNE_MERKLE_SUB_SPREAD, value);
        return STWO_OK;
    }
    if (n == "fft_max_strided_layers") {
        STWO_REQUIRE(value >= 4 && value <= 10, STWO_ERR_INVALID_ARGUMENT, "fft_max_strided_layers must be 4..10");
        set_tunable(TUNE_FFT_MAX_STRIDED, value);
        return STWO_OK;
    }
    if (n == "eval_at_point_groups_log") {
        STWO_REQUIRE(value == 0 || (value >= 2 && value <= 4), STWO_ERR_INVALID_ARGUMENT,
                     "eval_at_point_groups_log must be 0 (chosen per launch) or 2..4");
        set_tunable(TUNE_EAP_GROUPS_LOG, value);
        return STWO_OK;
    }
    if (n == "composition_tensor_cores") {
        STWO_REQUIRE(value == 0 || value == 1, STWO_ERR_INVALID_ARGUMENT, "composition_tensor_cores must be 0 or 1");
        set_tunable(TUNE_COMP_TENSOR, value);
        return STWO_OK;
    }
    if (n == "quotients_tensor_cores") {
        STWO_REQUIRE(value >= 0 && value <= 2, STWO_ERR_INVALID_ARGUMENT, "quotients_tensor_cores must be 0, 1 or 2");
        set_tunable(TUNE_QUOT_TENSOR, value);
        return STWO_OK;
    }
    return set_error(STWO_ERR_INVALID_ARGUMENT, "unknown tunable %s", name);
}

int stwo_probe_m31_butterflies(uint32_t iters, uint32_t *sink, uint64_t sink_words, uint64_t *butterflies,
                                void *stream) {
    return butterfly_probe_async(iters, sink, sink_words, butterflies, as_stream(stream));
}

int stwo_autotune(char *report, size_t report_cap) {
    cudaStream_t st = nullptr;
    STWO_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::string rep = "{";
    int rc = STWO_OK;
    {
        Buffers buf(st);
        // ---- FFT: 8 columns, interpolate at 2^L, evaluate at 2^(L+2)
        const uint32_t NCOL = 8;
        struct Case {
            uint32_t L;
            Tunable t;
            const char *name;
            int candidates[3];
        };
        const Case cases[] = {{18, TUNE_FFT_EPT_CONTIG_SMALL, "fft_ept_contig_small", {6, 5, 0}},
                              {22, TUNE_FFT_EPT_CONTIG_LARGE, "fft_ept_contig_large", {6, 5, 0}},
                              {22, TUNE_FFT_EPT_STRIDED, "fft_ept_strided", {6, 5, 0}},
                              {22, TUNE_FFT_MAX_STRIDED, "fft_max_strided_layers", {10, 7, 5}}};
        const uint32_t Dmax = 24;
        const uint64_t tsz = 1ull << (Dmax - 1);
        uint32_t *tw = buf.get(tsz), *itw = buf.get(tsz);
        STWO_REQUIRE(tw && itw, STWO_ERR_OUT_OF_MEMORY, "autotune allocation failed");
        rc = stwo_precompute_twiddles(1u << (30 - Dmax), (uint32_t)((1ull << (32 - Dmax)) & 0x7fffffffu), Dmax - 1,
                                      tw, itw, st);
        std::vector<uint32_t *> in(NCOL), out(NCOL);
        for (uint32_t c = 0; rc == STWO_OK && c < NCOL; c++) {
            in[c] = buf.get(1ull << 22);
            out[c] = buf.get(1ull << 24);
            STWO_REQUIRE(in[c] && out[c], STWO_ERR_OUT_OF_MEMORY, "autotune allocation failed");
            fill_kernel<<<1024, 256, 0, st>>>(in[c], 1ull << 22, c);
        }
        for (const Case &cs : cases) {
            if (rc) break;
            float best_ms = 1e30f;
            int best = tunable(cs.t);
            char part[128];
            std::string times;
            for (int v : cs.candidates) {
                if (v == 0) break;
                set_tunable(cs.t, v);
                float ms = 0;
                rc = time_best(st, [&] {
                    int r = fft_columns(in.data(), in.data(), NCOL, cs.L, cs.L, itw, tsz, true, st);
                    if (r) return r;
                    std::vector<const uint32_t *> src(in.begin(), in.end());
                    return fft_columns(src.data(), out.data(), NCOL, cs.L + 2, cs.L, tw, tsz, false, st);
                }, &ms);
                if (rc) break;
                snprintf(part, sizeof(part), "%s\"%d\": %.4f", times.empty() ? "" : ", ", v, ms);
                times += part;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = v;
                }
            }
            set_tunable(cs.t, best);
            snprintf(part, sizeof(part), "\"%s\": {\"chosen\": %d, \"ms\": {", cs.name, best);
            rep += (rep.size() > 1 ? ", " : "") + std::string(part) + times + "}}";
        }
        // ---- Merkle: 64 columns x 2^19 leaves, the whole tree
        if (rc == STWO_OK) {
            const uint32_t LOG = 19, NC = 64;
            std::vector<const uint32_t *> cols(NC);
            for (uint32_t c = 0; c < NC; c++) cols[c] = c < NCOL ? in[c] : in[c % NCOL] + ((c / NCOL) << LOG) % (1u << 22);
            uint32_t *table = buf.get(NC * 2);
            std::vector<uint32_t *> layers(LOG + 1);
            for (uint32_t l = 0; l <= LOG; l++) layers[l] = buf.get(8ull << l);
            uint32_t *tickets = buf.get(TICKETS);  // the tree kernel's, zeroed once
            STWO_REQUIRE(table && layers[LOG] && tickets, STWO_ERR_OUT_OF_MEMORY, "autotune allocation failed");
            STWO_CUDA_TRY(cudaMemsetAsync(tickets, 0, TICKETS * sizeof(uint32_t), st));
            STWO_CUDA_TRY(cudaMemcpyAsync(table, cols.data(), NC * sizeof(void *), cudaMemcpyHostToDevice, st));
            std::vector<const uint32_t *const *> lt(LOG + 1, nullptr);
            std::vector<uint32_t> ln(LOG + 1, 0);
            lt[LOG] = reinterpret_cast<const uint32_t *const *>(table);
            ln[LOG] = NC;
            float best_ms = 1e30f;
            int best = tunable(TUNE_MERKLE_SUB_THREADS);
            std::string times;
            char part[128];
            for (int v : {256, 128, 512}) {
                set_tunable(TUNE_MERKLE_SUB_THREADS, v);
                float ms = 0;
                rc = time_best(
                    st,
                    [&] {
                        return merkle_tree_dev_async(LOG, lt.data(), ln.data(), layers.data(), tickets, TICKETS, 1, 0, st);
                    },
                    &ms);
                if (rc) break;
                snprintf(part, sizeof(part), "%s\"%d\": %.4f", times.empty() ? "" : ", ", v, ms);
                times += part;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = v;
                }
            }
            set_tunable(TUNE_MERKLE_SUB_THREADS, best);
            snprintf(part, sizeof(part), ", \"merkle_sub_threads\": {\"chosen\": %d, \"ms\": {", best);
            rep += std::string(part) + times + "}}";
        }
        // ---- Merkle nodes per thread: 4 columns x 2^20 leaves (one compression per
        // leaf, the shape of the composition and FRI trees), the whole tree
        if (rc == STWO_OK) {
            const uint32_t LOG = 20, NC = 4;
            std::vector<const uint32_t *> cols(in.begin(), in.begin() + NC);
            uint32_t *table = buf.get(NC * 2);
            std::vector<uint32_t *> layers(LOG + 1);
            for (uint32_t l = 0; l <= LOG; l++) layers[l] = buf.get(8ull << l);
            uint32_t *tickets = buf.get(TICKETS);  // the tree kernel's, zeroed once
            STWO_REQUIRE(table && layers[LOG] && tickets, STWO_ERR_OUT_OF_MEMORY, "autotune allocation failed");
            STWO_CUDA_TRY(cudaMemsetAsync(tickets, 0, TICKETS * sizeof(uint32_t), st));
            STWO_CUDA_TRY(cudaMemcpyAsync(table, cols.data(), NC * sizeof(void *), cudaMemcpyHostToDevice, st));
            std::vector<const uint32_t *const *> lt(LOG + 1, nullptr);
            std::vector<uint32_t> ln(LOG + 1, 0);
            lt[LOG] = reinterpret_cast<const uint32_t *const *>(table);
            ln[LOG] = NC;
            float best_ms = 1e30f;
            int best = tunable(TUNE_MERKLE_SUB_SPREAD);
            std::string times;
            char part[128];
            for (int v : {3, 1, 2, 4, 5}) {
                set_tunable(TUNE_MERKLE_SUB_SPREAD, v);
                float ms = 0;
                rc = time_best(
                    st,
                    [&] {
                        return merkle_tree_dev_async(LOG, lt.data(), ln.data(), layers.data(), tickets, TICKETS, 1, 0, st);
                    },
                    &ms);
                if (rc) break;
                snprintf(part, sizeof(part), "%s\"%d\": %.4f", times.empty() ? "" : ", ", v, ms);
                times += part;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = v;
                }
            }
            set_tunable(TUNE_MERKLE_SUB_SPREAD, best);
            snprintf(part, sizeof(part), ", \"merkle_sub_spread\": {\"chosen\": %d, \"ms\": {", best);
            rep += std::string(part) + times + "}}";
        }
    }
    cudaStreamDestroy(st);
    rep += "}";
    if (report && report_cap) {
        strncpy(report, rep.c_str(), report_cap - 1);
        report[report_cap - 1] = 0;
    }
    return rc;
}

}  // extern "C"
