// yz_tc.cuh -- the sm_100a tensor-core primitives of the learned
// preconditioner's convolutions: shared-memory matrix descriptors,
// tcgen05.mma (kind::f16, BF16 operands, FP32 accumulator in TMEM), its
// commit to an mbarrier, TMEM allocation and the TMEM -> register load.
//
// Operand layout (both operands K-major, no swizzle): a "core matrix" is 8
// rows of 16 bytes (8 bf16 along K), stored contiguously (128 B).  A
// descriptor gives the start of the first core matrix, the byte distance
// between core matrices adjacent along K (LBO) and along M or N (SBO).  The
// kernels here keep each 8-element K chunk of a tile as rows at a 16-byte
// pitch, so SBO = 128 and LBO = the chunk's size.
//
// Every wait on an mbarrier is bounded (a clock budget); a wait that runs out
// records an error in device memory and the kernel returns after freeing its
// TMEM.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace yz {
namespace tc {

__device__ __forceinline__ uint32_t SmemAddr(const void *p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

//  shared-memory matrix descriptor (tcgen05 "matrix descriptor"): start
//  address, leading (K) and stride (M/N) byte offsets, all in 16-byte units;
//  bits 46-47 the descriptor version of sm_100; base offset 0, no swizzle
__device__ __forceinline__ uint64_t SmemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
	uint64_t d = 0;
	d |= (uint64_t)((addr >> 4) & 0x3FFFu);
	d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
	d |= (uint64_t)1u << 46;
	return d;
}

//  instruction descriptor of kind::f16: D in FP32, A and B in BF16, both
//  K-major, no negation or sparsity; N in units of 8, M in units of 16
__host__ __device__ constexpr uint32_t IdescBf16(int M, int N)
{
	return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

//  D[tmem] (+)= A[smem] * B[smem]^T, one M x N x 16 step; issued by one thread
__device__ __forceinline__ void MmaBf16(uint32_t tmemD, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate)
{
	asm volatile(
	    "{\n\t"
	    ".reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
	    "}\n" ::"r"(tmemD),
	    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

//  arrive on the mbarrier once every tcgen05 operation this thread issued
//  before has completed
__device__ __forceinline__ void Commit(uint64_t *bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(SmemAddr(bar))
	             : "memory");
}

__device__ __forceinline__ void FenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void FenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
//  make this thread's generic-proxy shared-memory writes visible to the
//  tensor core's (async proxy) reads
__device__ __forceinline__ void FenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void BarInit(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count));
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool BarTryWait(uint64_t *bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile(
	    "{\n\t"
	    ".reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t"
	    "}\n"
	    : "=r"(ok)
	    : "r"(SmemAddr(bar)), "r"(parity)
	    : "memory");
	return ok != 0;
}

//  wait for the phase of the given parity to complete, at most `budget`
//  clock cycles; false when the budget ran out
__device__ __forceinline__ bool BarWait(uint64_t *bar, uint32_t parity, long long budget)
{
	const long long t0 = clock64();
	while(!BarTryWait(bar, parity))
		if(clock64() - t0 > budget) return false;
	return true;
}

//  16 bytes global -> shared without staging through registers (the
//  copies of a thread stay in flight together); valid false fills zeros
__device__ __forceinline__ void CpAsync16(void *smem, const void *gmem, bool valid)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(SmemAddr(smem)), "l"(gmem),
	             "r"(valid ? 16 : 0)
	             : "memory");
}
__device__ __forceinline__ void CpAsyncWaitAll()
{
	asm volatile("cp.async.commit_group;" ::: "memory");
	asm volatile("cp.async.wait_group 0;" ::: "memory");
}

//  TMEM: one whole warp allocates `ncols` columns (a power of two, 32..512)
//  and writes their address to shared memory; the same warp frees them
__device__ __forceinline__ void TmemAlloc(uint32_t *slot, uint32_t ncols)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(slot)),
	             "r"(ncols));
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void TmemDealloc(uint32_t taddr, uint32_t ncols)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

//  16 consecutive FP32 columns of this thread's TMEM lane (a warp reads the
//  32 lanes of its sub-partition: warp w % 4 reads lanes 32 (w % 4) ..)
__device__ __forceinline__ void TmemLoad16(uint32_t taddr, float (&v)[16])
{
	uint32_t r[16];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
	    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	    : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for(int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

} // namespace tc
} // namespace yz
