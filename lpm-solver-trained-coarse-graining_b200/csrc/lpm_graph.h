// Replay of blocks of CG iterations as CUDA graphs, shared by the CG engines.
//
// A block of `poll` iterations depends only on buffers, sizes and options (the iteration number lives in device
// memory and is advanced by the last kernel of each iteration), so it is captured once and replayed for every later
// block with the same key.  Capture runs on a private non-blocking stream (the caller's stream may be the legacy
// default stream, which cannot be captured); the graph is launched on the caller's stream.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>

namespace lpm {

struct GraphKey {
    std::array<const void*, 10> ptr{};
    std::array<long long, 16> val{};
    long long waits = 0;  // the wait bounds baked into the captured launches (filled in by run_iteration_block)
    bool operator<(const GraphKey& o) const
    {
        return ptr != o.ptr ? ptr < o.ptr : (val != o.val ? val < o.val : waits < o.waits);
    }
};

unsigned tma_wait_polls();  // current poll bound of the TMA operators' data waits (kmv_tma.cu)

cudaGraphExec_t graph_find(const GraphKey& k);
void graph_put(const GraphKey& k, cudaGraphExec_t e);
cudaStream_t graph_capture_stream();
// Captures so far, graphs held now and evictions from the bounded cache (process-wide counters).
void graph_stats(long long* captures, long long* entries, long long* flushes);

// Runs `block` iterations starting at iteration `it`: replays (capturing on first use) the graph of `key` when
// use_graph, else launches eagerly.  one_iter(it, stream) issues one iteration's kernels and returns the launch status.
template <class F>
cudaError_t run_iteration_block(bool use_graph, const GraphKey& key, int it, int block, cudaStream_t st, F&& one_iter)
{
    if (!use_graph) {
        for (int b = 0; b < block; ++b) {
            const cudaError_t e = one_iter(it + b, st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    // a captured launch keeps the wait bound it was captured with: graphs of different bounds are different graphs
    GraphKey k = key;
    k.waits = (long long)tma_wait_polls();
    cudaGraphExec_t ge = graph_find(k);
    if (!ge) {
        cudaStream_t cs = graph_capture_stream();
        if (!cs) return cudaErrorNotReady;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        cudaError_t ce = cudaSuccess;
        for (int b = 0; b < block && ce == cudaSuccess; ++b) ce = one_iter(it + b, cs);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(cs, &g);
        if (ce != cudaSuccess || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return ce != cudaSuccess ? ce : e;
        }
        e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return e;
        graph_put(k, ge);
    }
    return cudaGraphLaunch(ge, st);
}

}  // namespace lpm
