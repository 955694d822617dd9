// kb_umma.cu -- a plain BF16 GEMM on the tcgen05 engines (kb_umma.cuh,
// kb_umma_tma.cuh) that exercises both operand majors; the tests use it to pin
// the shared-memory descriptors that the convolutions of the warm-start
// network rely on.  Also the tensor-map encoder of the TMA engine.
#include "kb_common.cuh"
#include "kb_umma_tma.cuh"

namespace kb {
namespace umma {

static int g_engine = 2;
int engine() { return g_engine; }
void set_engine(int e) { g_engine = e; }

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

int bf16_map(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims,
             const cuuint64_t *strides, const cuuint32_t *box, int swz, const char *what) {
    if (!encode_fn()) return kb::set_error(KB_ERR_CUDA, "%s: cuTensorMapEncodeTiled unavailable", what);
    if ((uintptr_t)base % 16) return kb::set_error(KB_ERR_ARG, "%s: tensor base not 16-byte aligned", what);
    const CUtensorMapSwizzle sw = swz == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                  : swz == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                              : CU_TENSOR_MAP_SWIZZLE_32B;
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    const CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank,
                                   const_cast<void *>(base), dims, strides, box, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return kb::set_error(KB_ERR_CUDA, "%s: cuTensorMapEncodeTiled failed (%d)", what, (int)r);
    return 0;
}

int pick_bn(int n) {
    for (int bn = NT; bn >= 16; bn -= 16)
        if (n % bn == 0) return bn;
    return 0;
}

}  // namespace umma
}  // namespace kb

extern "C" int kb_gemm_bf16(const void *A, const void *B, float *C, int M, int N, int K, int a_mn,
                            int b_mn, int *err_device, void *stream) {
    using namespace kb::umma;
    KB_REQUIRE(A && B && C && err_device, "kb_gemm_bf16: null pointer");
    KB_REQUIRE(M > 0 && M % BM == 0, "kb_gemm_bf16: M=%d must be a positive multiple of 128", M);
    KB_REQUIRE(K > 0 && K % BK == 0, "kb_gemm_bf16: K=%d must be a positive multiple of 64", K);
    const int bn = pick_bn(N);
    KB_REQUIRE(N > 0 && bn > 0, "kb_gemm_bf16: N=%d must be a positive multiple of 16", N);
    KB_REQUIRE(((uintptr_t)A % 16) == 0 && ((uintptr_t)B % 16) == 0 && ((uintptr_t)C % 16) == 0,
               "kb_gemm_bf16: A, B and C must be 16-byte aligned");
    const dim3 grid(M / BM, N / bn);
    const __nv_bfloat16 *a = (const __nv_bfloat16 *)A, *b = (const __nv_bfloat16 *)B;
    cudaStream_t st = kb::as_stream(stream);
    int rc;
    if (engine() == 2) {
        // TMA-staged engine: A and B boxes with 128-byte swizzle (B MN-major:
        // the widest swizzle whose run divides bn)
        const int eb = chunk_of(bn);
        CUtensorMap ma, mb;
        const char *what = "kb_gemm_bf16";
        if (!a_mn) {
            const cuuint64_t d[2] = {(cuuint64_t)K, (cuuint64_t)M}, sd[1] = {(cuuint64_t)K * 2};
            const cuuint32_t bx[2] = {64, 128};
            if ((rc = bf16_map(&ma, A, 2, d, sd, bx, 128, what))) return rc;
        } else {
            const cuuint64_t d[2] = {(cuuint64_t)M, (cuuint64_t)K}, sd[1] = {(cuuint64_t)M * 2};
            const cuuint32_t bx[2] = {64, 64};
            if ((rc = bf16_map(&ma, A, 2, d, sd, bx, 128, what))) return rc;
        }
        if (!b_mn) {
            const cuuint64_t d[2] = {(cuuint64_t)K, (cuuint64_t)N}, sd[1] = {(cuuint64_t)K * 2};
            const cuuint32_t bx[2] = {64, (cuuint32_t)bn};
            if ((rc = bf16_map(&mb, B, 2, d, sd, bx, 128, what))) return rc;
        } else {
            const cuuint64_t d[2] = {(cuuint64_t)N, (cuuint64_t)K}, sd[1] = {(cuuint64_t)N * 2};
            const cuuint32_t bx[2] = {(cuuint32_t)eb, 64};
            if ((rc = bf16_map(&mb, B, 2, d, sd, bx, 2 * eb, what))) return rc;
        }
        const uint32_t ab = BM * BK * 2, bb = round1k((uint32_t)bn * BK * 2);
        auto go = [&](auto op) {
            op.ma = ma;
            op.mb = mb;
            op.c = C;
            op.M = M;
            op.N = N;
            op.K = K;
            op.bn = bn;
            op.eb = eb;
            op.nb = bn / eb;
            op.a_bytes = ab;
            op.b_bytes = bb;
            op.res_bytes = 0;
            op.acc_cols = tmem_cols(bn);
            op.nbuf = 2;
            op.ncols = bn;
            op.cps = tma_fit(op);
            return launch_tma(op, grid, err_device, st);
        };
        if (!a_mn && !b_mn) rc = go(GemmTma<false, false>{});
        else if (a_mn && b_mn) rc = go(GemmTma<true, true>{});
        else if (a_mn) rc = go(GemmTma<true, false>{});
        else rc = go(GemmTma<false, true>{});
    } else if (!a_mn && !b_mn) rc = launch(GemmOp<false, false>{a, b, C, M, N, K, bn}, grid, err_device, st);
    else if (a_mn && b_mn) rc = launch(GemmOp<true, true>{a, b, C, M, N, K, bn}, grid, err_device, st);
    else if (a_mn) rc = launch(GemmOp<true, false>{a, b, C, M, N, K, bn}, grid, err_device, st);
    else rc = launch(GemmOp<false, true>{a, b, C, M, N, K, bn}, grid, err_device, st);
    if (rc) return rc;
    return kb::check_launch("kb_gemm_bf16");
}
