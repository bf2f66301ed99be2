// warmstart.cu -- kernels of the learned warm start: the tensor-core matrix
// product (umma_gemm.cuh) behind a C ABI entry.
#include <cuda_runtime.h>

#include <string>

#include "../../include/tangle_cuda.h"
#include "umma_gemm.cuh"

namespace tgl {
void set_last_error(const std::string &message);
}

namespace {

int gemm_error(int code, const std::string &message) {
    tgl::set_last_error(message);
    return code;
}

}  // namespace

extern "C" int tgl_gemm_bf16(const tgl_gemm *p, void *stream) {
    if (!p || !p->a || !p->b || (!p->out_f32 && !p->out_bf16))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: null argument");
    if (p->n < 16 || p->n > 256 || p->n % 16 || p->m < 0 || p->k < 0)
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: n must be a multiple of 16 in [16, 256]");
    if (((!p->a_mn || !p->b_mn) && p->k % 8) || (p->a_mn && p->lda % 8) || (p->b_mn && p->ldb % 8) ||
        (!p->a_mn && p->lda % 8) || (!p->b_mn && p->ldb % 8))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: leading dimensions (and K with a K-major operand) "
                                           "must be multiples of 8 elements");
    if ((p->a_mn ? p->lda < p->m : p->lda < p->k) || (p->b_mn ? p->ldb < p->n : p->ldb < p->k) ||
        (p->out_f32 && p->ldo < p->n) || (p->out_bf16 && p->ldo_bf16 < p->n))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: a leading dimension is shorter than its rows");
    if ((reinterpret_cast<uintptr_t>(p->a) | reinterpret_cast<uintptr_t>(p->b)) & 15)
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: operands must be 16-byte aligned");
    if (p->out_f32 && (p->ldo % 4 || (reinterpret_cast<uintptr_t>(p->out_f32) & 15)))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: f32 output must be 16-byte aligned with ldo % 4 == 0");
    if (p->out_bf16 && (p->ldo_bf16 % 8 || (reinterpret_cast<uintptr_t>(p->out_bf16) & 15)))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: bf16 output must be 16-byte aligned with ldo % 8 == 0");
    const int64_t k_split = p->k_split > 0 ? p->k_split : (p->k > 0 ? p->k : 1);
    if (p->k_split > 0 && (p->k_split % 64 || p->bias || p->relu || p->out_bf16))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: split K needs k_split % 64 == 0 and a plain f32 output");
    if (p->m == 0) return 0;
    tgl::GemmArgs g{};
    g.a = reinterpret_cast<const __nv_bfloat16 *>(p->a);
    g.b = reinterpret_cast<const __nv_bfloat16 *>(p->b);
    g.lda = p->lda;
    g.ldb = p->ldb;
    g.m = p->m;
    g.n = p->n;
    g.k = p->k;
    g.a_mn = p->a_mn ? 1 : 0;
    g.b_mn = p->b_mn ? 1 : 0;
    g.k_split = k_split;
    g.bias = p->bias;
    g.relu = p->relu ? 1 : 0;
    g.out_f32 = p->out_f32;
    g.ldo = p->ldo;
    g.out_bf16 = reinterpret_cast<__nv_bfloat16 *>(p->out_bf16);
    g.ldo_bf16 = p->ldo_bf16;
    g.error = p->error;
    const int64_t splits = p->k > 0 ? (p->k + k_split - 1) / k_split : 1;
    if (splits > 65535) return gemm_error(TGL_ERR_UNSUPPORTED, "tgl_gemm_bf16: too many K splits");
    const size_t smem = (size_t)tgl::GEMM_BM * tgl::GEMM_KC * 2 + (size_t)p->n * tgl::GEMM_KC * 2;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(tgl::umma_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((size_t)tgl::GEMM_BM * tgl::GEMM_KC * 2 + 256 * tgl::GEMM_KC * 2));
        configured = true;
    }
    dim3 grid((unsigned)((p->m + tgl::GEMM_BM - 1) / tgl::GEMM_BM), (unsigned)splits);
    tgl::umma_gemm_kernel<<<grid, tgl::GEMM_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(g);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return gemm_error(TGL_ERR_CUDA, std::string("tgl_gemm_bf16: ") + cudaGetErrorString(e));
    return 0;
}
