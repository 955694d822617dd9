// kb_graph.cu -- CUDA-graph capture of a sequence of library calls, and the
// bounded-wait self test.
//
// persistent_fused_bgk! / persistent_aa_bgk! (src/kernels/persistent_bgk_2d.jl:
// 17-56) queue Nt launches from the host with one synchronise at the end.
// Here the caller captures the launches of one (or many) steps once and
// replays the instantiated graph, which removes the per-launch host cost that
// dominates small grids.
#include <new>

#include "kb_common.cuh"

struct kb_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace kb {

// Spin until *word != old or `limit` polls have passed; on time-out set *err.
// The same bounded wait guards the grid barrier of the batched kernel.
__device__ __forceinline__ bool bounded_wait_change(volatile unsigned *word, unsigned old,
                                                    long long limit, int *err) {
    long long it = 0;
    while (*word == old) {
        if (++it > limit) {
            atomicExch(err, 1);
            return false;
        }
        __nanosleep(128);
    }
    return true;
}

__global__ void wait_selftest_k(unsigned *word, long long limit, int *err, long long *polls) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const bool ok = bounded_wait_change(word, *word, limit, err);
        *polls = ok ? 0 : limit;
    }
}

}  // namespace kb

extern "C" {

int kb_graph_begin(void *stream) {
    KB_REQUIRE(stream, "kb_graph_begin: capture needs a non-default stream");
    cudaError_t e = cudaStreamBeginCapture(kb::as_stream(stream), cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
        return kb::set_error(KB_ERR_CUDA, "kb_graph_begin: %s", cudaGetErrorString(e));
    return KB_OK;
}

int kb_graph_end(void *stream, kb_graph **out) {
    KB_REQUIRE(stream && out, "kb_graph_end: null pointer");
    kb_graph *g = new (std::nothrow) kb_graph();
    if (!g) return kb::set_error(KB_ERR_NOMEM, "kb_graph_end: out of host memory");
    cudaError_t e = cudaStreamEndCapture(kb::as_stream(stream), &g->graph);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) {
        if (g->graph) cudaGraphDestroy(g->graph);
        delete g;
        cudaGetLastError();
        return kb::set_error(KB_ERR_CUDA, "kb_graph_end: %s", cudaGetErrorString(e));
    }
    *out = g;
    return KB_OK;
}

int kb_graph_launch(kb_graph *g, void *stream) {
    KB_REQUIRE(g && g->exec, "kb_graph_launch: null graph");
    cudaError_t e = cudaGraphLaunch(g->exec, kb::as_stream(stream));
    if (e != cudaSuccess)
        return kb::set_error(KB_ERR_CUDA, "kb_graph_launch: %s", cudaGetErrorString(e));
    return KB_OK;
}

int kb_graph_destroy(kb_graph *g) {
    if (!g) return KB_OK;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return KB_OK;
}

int kb_selftest_bounded_wait(long long limit, int *timed_out, void *stream) {
    KB_REQUIRE(timed_out, "kb_selftest_bounded_wait: null pointer");
    KB_REQUIRE(limit > 0 && limit <= (1ll << 24), "kb_selftest_bounded_wait: limit out of range");
    cudaStream_t s = kb::as_stream(stream);
    void *buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, 64, s);
    if (e != cudaSuccess) return kb::set_error(KB_ERR_NOMEM, "kb_selftest_bounded_wait: %s", cudaGetErrorString(e));
    e = cudaMemsetAsync(buf, 0, 64, s);
    unsigned *word = (unsigned *)buf;
    int *err = (int *)((char *)buf + 16);
    long long *polls = (long long *)((char *)buf + 32);
    if (e == cudaSuccess) {
        kb::wait_selftest_k<<<1, 32, 0, s>>>(word, limit, err, polls);
        e = cudaGetLastError();
    }
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(buf, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return kb::set_error(KB_ERR_CUDA, "kb_selftest_bounded_wait: %s", cudaGetErrorString(e));
    *timed_out = h;
    return h ? kb::set_error(KB_ERR_TIMEOUT, "kb_selftest_bounded_wait: wait ran out after %lld polls", limit)
             : KB_OK;
}

}  // extern "C"
