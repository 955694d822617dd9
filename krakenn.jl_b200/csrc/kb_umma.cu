// kb_umma.cu -- a plain BF16 GEMM on the tcgen05 mainloop (kb_umma.cuh) that
// exercises both operand majors; the tests use it to pin the shared-memory
// descriptors that the convolutions of the warm-start network rely on.
#include "kb_common.cuh"
#include "kb_umma.cuh"

namespace kb {
namespace umma {

static int g_engine = 1;  // measured faster: see engine()
int engine() { return g_engine; }
void set_engine(int e) { g_engine = e; }

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
    if (!a_mn && !b_mn) rc = launch(GemmOp<false, false>{a, b, C, M, N, K, bn}, grid, err_device, st);
    else if (a_mn && b_mn) rc = launch(GemmOp<true, true>{a, b, C, M, N, K, bn}, grid, err_device, st);
    else if (a_mn) rc = launch(GemmOp<true, false>{a, b, C, M, N, K, bn}, grid, err_device, st);
    else rc = launch(GemmOp<false, true>{a, b, C, M, N, K, bn}, grid, err_device, st);
    if (rc) return rc;
    return kb::check_launch("kb_gemm_bf16");
}
