// Tensor-core issue rate of the MMA shapes a DFT-as-matrix-product stage can use: one CTA per SM
// issues 1024 tcgen05.mma.kind::f16 (BF16 in, FP32 accumulate in tensor memory, K = 16, both
// operands K-major in shared memory) from one thread and times them to completion with clock64;
// prints cycles per instruction and MACs per cycle per SM for M in {64, 128}, N in {64..256},
// one or several independent accumulators, two operand layouts (no swizzle, 128-byte swizzle),
// and two ways of issuing (descriptors formed per MMA in a loop, or formed once with the K steps
// unrolled).  The first shape is also checked against a host product.  Standalone program, not
// part of the library:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o umma_rate umma_rate.cu && ./umma_rate
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <vector>

namespace {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// byte offset of element (r, k), K = 64 (8 chunks of 8): 0 = no swizzle (LBO 128, SBO 1024),
// 1 = 128-byte swizzle (SBO 1024, chunk index XOR row within the 8-row atom)
__device__ __forceinline__ int elem_off(int layout, int r, int k) {
    const int c = k >> 3, e = (k & 7) * 2;
    return layout == 0 ? (r >> 3) * 1024 + c * 128 + (r & 7) * 16 + e : (r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4) + e;
}

__device__ __forceinline__ uint64_t make_desc(int layout, uint32_t addr, int kstep) {
    const uint32_t start = layout == 0 ? addr + kstep * 256 : addr + kstep * 32;
    const uint32_t lbo = layout == 0 ? 128 : 16, sbo = 1024;
    return (uint64_t)((start >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | ((uint64_t)1 << 46) | ((uint64_t)(layout == 0 ? 0 : 2) << 61);
}

constexpr int kReps = 256;   // x 4 K steps = 1024 MMAs per CTA

__global__ void __launch_bounds__(128, 1)
umma_rate_kernel(const uint16_t* A, const uint16_t* B, float* D, int layout, int M, int N, int nacc, int fast,
                 int* err, unsigned long long* cycles) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, w = tid / 32;
    unsigned char* As = sm;            // 128 x 64 BF16 (16 KB)
    unsigned char* Bs = sm + 16384;    // 256 x 64 BF16 (32 KB)
    if ((saddr(sm) & 1023) != 0) {     // the swizzle atoms need 1024-byte alignment (uniform exit)
        if (tid == 0) atomicExch(err, 2);
        return;
    }
    for (int i = tid; i < 128 * 64; i += 128)
        *reinterpret_cast<uint16_t*>(As + elem_off(layout, i / 64, i % 64)) = A[i];
    for (int i = tid; i < 256 * 64; i += 128)
        *reinterpret_cast<uint16_t*>(Bs + elem_off(layout, i / 64, i % 64)) = B[i];
    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tbase)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tbase;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
    bool ok = true;
    for (int pass = 0; pass < 2 && ok; pass++) {   // pass 0: one product (checked); pass 1: timed
        const int reps = pass == 0 ? 1 : kReps;
        const unsigned long long t0 = clock64();
        if (tid == 0 && !fast) {
            for (int r = 0; r < reps; r++)
                for (int s = 0; s < 4; s++) {
                    const uint32_t acc = (r >= nacc || s > 0) ? 1u : 0u;
                    const uint32_t d = tmem + (uint32_t)((r % nacc) * N);
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
                        "l"(make_desc(layout, saddr(As), s)), "l"(make_desc(layout, saddr(Bs), s)), "r"(idesc), "r"(acc));
                }
        } else if (tid == 0) {
            // descriptors formed once, the four K steps unrolled, one accumulator
            uint64_t da[4], db[4];
            for (int s = 0; s < 4; s++) {
                da[s] = make_desc(layout, saddr(As), s);
                db[s] = make_desc(layout, saddr(Bs), s);
            }
            for (int r = 0; r < reps; r++) {
#pragma unroll
                for (int s = 0; s < 4; s++) {
                    const uint32_t acc = (r > 0 || s > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(da[s]), "l"(db[s]), "r"(idesc), "r"(acc));
                }
            }
        }
        if (tid == 0)
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(&mbar))
                         : "memory");
        ok = false;
        const unsigned long long g0 = now_ns();
        for (long long i = 0; i < (1ll << 22); i++) {   // bounded: 200 ms or 4M polls
            uint32_t done;
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(saddr(&mbar)), "r"(pass)
                : "memory");
            if (done) { ok = true; break; }
            if ((i & 1023) == 1023 && now_ns() - g0 > 200000000ull) break;
        }
        const unsigned long long t1 = clock64();
        if (!ok) atomicExch(err, 1);
        if (tid == 0 && pass == 1) atomicAdd(cycles, t1 - t0);
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (ok && pass == 0 && blockIdx.x == 0 && M == 128) {
            for (int c0 = 0; c0 < 64; c0 += 32) {
                uint32_t r[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                      "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                      "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(tmem + ((uint32_t)(w * 32) << 16) + c0));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                for (int j = 0; j < 32; j++) D[tid * 64 + c0 + j] = __uint_as_float(r[j]);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

uint16_t to_bf16(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}
float from_bf16(uint16_t h) {
    const uint32_t u = (uint32_t)h << 16;
    float x;
    memcpy(&x, &u, 4);
    return x;
}

}  // namespace

int main() {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    std::vector<uint16_t> a(128 * 64), b(256 * 64);
    srand(3);
    for (auto& x : a) x = to_bf16((float)rand() / RAND_MAX - 0.5f);
    for (auto& x : b) x = to_bf16((float)rand() / RAND_MAX - 0.5f);
    uint16_t *dA, *dB;
    float* dD;
    int* dErr;
    unsigned long long* dCyc;
    cudaMalloc(&dA, a.size() * 2);
    cudaMalloc(&dB, b.size() * 2);
    cudaMalloc(&dD, 128 * 64 * 4);
    cudaMalloc(&dErr, 4);
    cudaMalloc(&dCyc, 8);
    cudaMemcpy(dA, a.data(), a.size() * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, b.data(), b.size() * 2, cudaMemcpyHostToDevice);
    const int smem = 16384 + 32768;
    cudaFuncSetAttribute(umma_rate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    struct Shape { int M, N, nacc, fast; };
    const Shape shapes[] = {{128, 64, 1, 0}, {128, 64, 4, 0}, {128, 96, 1, 0}, {128, 128, 1, 0}, {128, 128, 2, 0},
                            {128, 256, 1, 0}, {128, 256, 2, 0}, {64, 64, 1, 0}, {64, 256, 1, 0},
                            {128, 64, 1, 1}, {128, 96, 1, 1}, {128, 128, 1, 1}, {128, 256, 1, 1}};
    printf("layout     M    N  accumulators  issue     cycles/MMA  MAC/cycle/SM (peak 4096)  check\n");
    int rc = 0;
    for (int layout = 0; layout < 2 && rc == 0; layout++)
        for (const Shape& s : shapes) {
            std::vector<float> d(128 * 64, 0.f);
            cudaMemset(dD, 0, 128 * 64 * 4);
            cudaMemset(dErr, 0, 4);
            cudaMemset(dCyc, 0, 8);
            umma_rate_kernel<<<sms, 128, smem>>>(dA, dB, dD, layout, s.M, s.N, s.nacc, s.fast, dErr, dCyc);
            const cudaError_t e = cudaDeviceSynchronize();
            int err = 0;
            unsigned long long cyc = 0;
            cudaMemcpy(&err, dErr, 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(&cyc, dCyc, 8, cudaMemcpyDeviceToHost);
            cudaMemcpy(d.data(), dD, d.size() * 4, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess || err) {
                printf("failed: %s, status %d\n", cudaGetErrorString(e), err);
                rc = 1;
                break;
            }
            char check[32] = "";
            if (s.M == 128) {   // D = A B^T over K = 64 for N columns 0..63
                double worst = 0, scale = 0;
                for (int m = 0; m < 128; m++)
                    for (int n = 0; n < 64; n++) {
                        double ref = 0;
                        for (int k = 0; k < 64; k++) ref += (double)from_bf16(a[m * 64 + k]) * from_bf16(b[n * 64 + k]);
                        worst = fmax(worst, fabs(ref - d[m * 64 + n]));
                        scale = fmax(scale, fabs(ref));
                    }
                snprintf(check, sizeof(check), "%.1e", worst / scale);
                if (!(worst / scale < 1e-5)) rc = 2;
            }
            const double per = (double)cyc / sms / (kReps * 4);
            printf("%-9s %4d %4d  %12d  %-8s  %10.1f  %12.0f  %11s  %s\n", layout == 0 ? "no-swizzle" : "swizzle128", s.M,
                   s.N, s.nacc, s.fast ? "unrolled" : "loop", per, s.M * s.N * 16.0 / per, "", check);
        }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dErr);
    cudaFree(dCyc);
    return rc;
}
