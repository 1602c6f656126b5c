// Tensor-core cross-multiply-accumulate for sm_100a (tcgen05 + TMA).
//
// Core::processdata's XMAC (mpifxcorr/src/core.cpp:877-972) and the Mode
// autocorrelations (mode.cpp:1293-1369) per channel are V = X X^H, with X the
// [inputs x time] matrix of one channel's spectra.  With A = X written as real
// rows (2 rows per input: real and imaginary part, interleaved), A A^T holds
// every product: for inputs a, b
//     Re V[a][b] = P[2a][2b] + P[2a+1][2b+1],  Im V[a][b] = P[2a+1][2b] - P[2a][2b+1].
//
// The F stage writes the spectra as BF16 [chan][R2 real rows][Tpad times]
// (K-major, time contiguous).  G = floor(128 / R2) consecutive channels form
// one M = 128 operand tile (their R2-row blocks stacked, the rest of the 128
// rows belong to the next channels and only feed outputs that are discarded);
// one tcgen05.mma (kind::f16, M = 128, N = 128, K = 16) uses the same shared
// memory tile as A and B, so the G diagonal R2 x R2 blocks of the 128 x 128
// FP32 accumulator in tensor memory are the G channels' A A^T.  Tiles arrive by
// TMA (no multicast) with 128-byte swizzle into a 3-stage ring; one thread
// issues the TMA loads, one issues the MMAs, and all four warps run the
// epilogue (tcgen05.ld, recombination into complex products, accumulation
// into the [chan][output] accumulators).  Every wait is bounded: on timeout
// the CTA records an error code and still releases its tensor memory.

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

namespace {

constexpr int kStages = 3;
constexpr int kKTile = 64;            // times per stage (128 bytes of BF16 per row)
constexpr int kRowBytes = kKTile * 2;
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
	             : "memory");
}

// bounded wait for the phase with parity `parity` to complete; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
	const uint32_t a = smem_u32(bar);
	for(uint32_t it = 0; it < kWaitLimit; it++)
	{
		uint32_t done;
		asm volatile(
		    "{\n\t.reg .pred p;\n\t"
		    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		    "selp.u32 %0, 1, 0, p;\n\t}\n"
		    : "=r"(done)
		    : "r"(a), "r"(parity)
		    : "memory");
		if(done)
			return true;
	}
	return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
	asm volatile(
	    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
	        smem_u32(dst)),
	    "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
	    : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (version 1 = tcgen05)
__device__ __forceinline__ uint64_t make_sdesc(uint32_t saddr)
{
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3FFF);            // start address
	d |= (uint64_t)1 << 16;                             // leading byte offset (unused for swizzled K-major)
	d |= (uint64_t)(1024 >> 4) << 32;                   // stride byte offset
	d |= (uint64_t)1 << 46;                             // descriptor version
	d |= (uint64_t)2 << 61;                             // SWIZZLE_128B
	return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
	    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
	             : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v)
{
	uint32_t r[8];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
	             : "r"(taddr));
#pragma unroll
	for(int i = 0; i < 8; i++)
		v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

}  // namespace

struct TcParams {
	int32_t Tpad;           // times per channel row (multiple of 64)
	int32_t R2;             // real rows per channel (multiple of 8, <= 128)
	int32_t G;              // channels per 128-row tile
	int32_t NG;             // tiles per CTA
	int32_t boxrows;        // rows per TMA box ((NG-1)*G*R2 + 128)
	int32_t tmem_cols;      // tensor-memory columns allocated (power of two)
	int32_t *err;           // error flag (nonzero: a bounded wait expired)
};

// One CTA: NG tiles of G channels each, of the frequency plans[plan_idx[blockIdx.y]].
__global__ void __launch_bounds__(128, 1) k_xmac_tc(const __grid_constant__ CUtensorMap tmap,
                                                    const DevFreqPlan *__restrict__ plans,
                                                    const int32_t *__restrict__ plan_idx,
                                                    const int64_t *__restrict__ rowbase, TcParams tp,
                                                    float2 *__restrict__ acc)
{
	extern __shared__ __align__(1024) unsigned char smem_tc[];
	__shared__ uint64_t full_bar[kStages], empty_bar[kStages], done_bar;
	__shared__ uint32_t tmem_base_s;
	__shared__ int fail_s;
	__shared__ int issued_s, consumed_s;

	const int fidx = plan_idx[blockIdx.y];
	const DevFreqPlan P = plans[fidx];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int ch_per_cta = tp.NG * tp.G;
	const int c_first = blockIdx.x * ch_per_cta;
	if(c_first >= P.nchan)
		return;
	// 1024-aligned stage buffers (128-byte swizzle atoms)
	unsigned char *stage0 = (unsigned char *)(((uintptr_t)smem_tc + 1023) & ~(uintptr_t)1023);
	const int stage_bytes = ((tp.boxrows * kRowBytes) + 1023) & ~1023;
	const uint32_t tx_bytes = (uint32_t)(tp.boxrows * kRowBytes);
	const int nkb = tp.Tpad / kKTile;
	const int64_t row0 = rowbase[fidx] + (int64_t)c_first * tp.R2;

	if(threadIdx.x == 0)
	{
		for(int s = 0; s < kStages; s++)
		{
			mbar_init(&full_bar[s], 1);
			mbar_init(&empty_bar[s], 1);
		}
		mbar_init(&done_bar, 1);
		fail_s = 0;
		issued_s = 0;
		consumed_s = 0;
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	if(warp == 0)
	{
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_s)),
		             "r"((uint32_t)tp.tmem_cols));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
	}
	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	const uint32_t tmem = tmem_base_s;

	if(threadIdx.x == 0)
	{
		// TMA producer
		for(int kb = 0; kb < nkb; kb++)
		{
			const int s = kb % kStages;
			if(kb >= kStages && !mbar_wait(&empty_bar[s], ((kb / kStages) - 1) & 1))
			{
				fail_s = 1;
				break;
			}
			mbar_expect_tx(&full_bar[s], tx_bytes);
			tma_load_2d(stage0 + (size_t)s * stage_bytes, &tmap, kb * kKTile, (int)row0, &full_bar[s]);
			issued_s = kb + 1;
		}
	}
	else if(threadIdx.x == 32)
	{
		// MMA issuer: M = 128, N = 128, BF16 x BF16 -> FP32, A and B K-major
		const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
		for(int kb = 0; kb < nkb; kb++)
		{
			const int s = kb % kStages;
			if(!mbar_wait(&full_bar[s], (kb / kStages) & 1))
			{
				fail_s = 2;
				break;
			}
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			const uint32_t sbase = smem_u32(stage0 + (size_t)s * stage_bytes);
			for(int g = 0; g < tp.NG; g++)
			{
				const uint32_t tile = sbase + (uint32_t)(g * tp.G * tp.R2 * kRowBytes);
#pragma unroll
				for(int kk = 0; kk < kKTile / 16; kk++)
				{
					const uint64_t d = make_sdesc(tile + kk * 32);
					mma_bf16(tmem + (uint32_t)(g * 128), d, d, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
				}
			}
			mma_commit(&empty_bar[s]);
			consumed_s = kb + 1;
		}
		mma_commit(&done_bar);
	}
	__syncwarp();
	// epilogue: every thread owns tensor-memory lane (row) 32*warp + lane
	const bool okw = mbar_wait(&done_bar, 0);
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	__syncthreads();
	const int good = __syncthreads_and(okw && fail_s == 0);
	if(!good)
	{
		if(threadIdx.x == 0 && tp.err)
			atomicExch(tp.err, fail_s ? fail_s : 3);
	}
	else
	{
		// results of the CTA's channels: [channel][output] in shared memory
		// (the stage ring is idle: every load was consumed by an MMA)
		const int nout = P.acc_cstride;
		float2 *vbuf = (float2 *)stage0;
		const int nval = ch_per_cta * nout;
		for(int i = threadIdx.x; i < nval; i += blockDim.x)
			vbuf[i] = make_float2(0.0f, 0.0f);
		__syncthreads();
		const int row = 32 * warp + lane;
		const int nin = P.nrow;
		for(int g = 0; g < tp.NG; g++)
		{
			// channels of this tile touched by this warp's 32 rows
			const int qlo = (32 * warp) / tp.R2;
			const int qhi = min(tp.G - 1, (32 * warp + 31) / tp.R2);
			for(int q = qlo; q <= qhi; q++)
			{
				const int cl = g * tp.G + q;                 // channel within the CTA
				const bool mine = row >= q * tp.R2 && row < (q + 1) * tp.R2;
				const int r2 = row - q * tp.R2;
				float pv[128];
				for(int j8 = 0; j8 < tp.R2; j8 += 8)
					tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(g * 128 + q * tp.R2 + j8), pv + j8);
				tmem_ld_wait();
				const int a = r2 >> 1;
				const bool even = (r2 & 1) == 0;
				for(int b = 0; b < nin; b++)
				{
					const float p_e_re = pv[2 * b], p_e_im = pv[2 * b + 1];        // P[row][2b], P[row][2b+1]
					const float o_re = __shfl_xor_sync(0xffffffffu, p_e_re, 1);    // partner's P[.][2b]
					const float o_im = __shfl_xor_sync(0xffffffffu, p_e_im, 1);    // partner's P[.][2b+1]
					if(!mine || !even || a >= nin || b < a)
						continue;
					const float vre = p_e_re + o_im;          // P[2a][2b] + P[2a+1][2b+1]
					const float vim = o_re - p_e_im;          // P[2a+1][2b] - P[2a][2b+1]
					const int dA = P.destA[a * nin + b];
					const int dB = P.destB[a * nin + b];
					if(dA >= 0)
						vbuf[cl * nout + dA] = make_float2(vre, vim);
					if(dB >= 0)
						vbuf[cl * nout + dB] = make_float2(vre, -vim);
				}
			}
		}
		__syncthreads();
		// coalesced accumulate into the contiguous [channel][output] block
		const int nvalid = min(ch_per_cta, P.nchan - c_first) * nout;
		float2 *dst = acc + P.acc_off + (int64_t)c_first * nout;
		for(int i = threadIdx.x; i < nvalid; i += blockDim.x)
		{
			const float2 v = vbuf[i], o = dst[i];
			dst[i] = make_float2(o.x + v.x, o.y + v.y);
		}
	}
	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	if(threadIdx.x == 0)
	{
		// on the error path, wait (bounded) for TMA loads nobody consumed
		for(int kb = consumed_s; kb < issued_s; kb++)
			mbar_wait(&full_bar[kb % kStages], (kb / kStages) & 1);
	}
	__syncthreads();
	if(warp == 0)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)tp.tmem_cols));
}

// ---------------------------------------------------------------- host side
typedef CUresult (*PFN_encodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                     const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

bool tc_make_tensormap(void *map_out, const void *spec_bf16, int64_t total_rows, int Tpad, int boxrows)
{
	if(((uintptr_t)map_out & 63) != 0)
		return false;                // CUtensorMap must be 64-byte aligned
	static PFN_encodeTiled encode = nullptr;
	if(!encode)
	{
		void *fn = nullptr;
		cudaDriverEntryPointQueryResult q;
		if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
		   q != cudaDriverEntryPointSuccess || !fn)
			return false;
		encode = (PFN_encodeTiled)fn;
	}
	// the TMA x coordinate (time) is always a multiple of 64 elements = 128 bytes
	cuuint64_t dims[2] = {(cuuint64_t)Tpad, (cuuint64_t)total_rows};
	cuuint64_t strides[1] = {(cuuint64_t)Tpad * 2};
	cuuint32_t box[2] = {(cuuint32_t)kKTile, (cuuint32_t)boxrows};
	cuuint32_t estr[2] = {1, 1};
	CUresult r = encode((CUtensorMap *)map_out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)spec_bf16, dims, strides,
	                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
	                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	return r == CUDA_SUCCESS;
}

size_t tc_tensormap_size() { return sizeof(CUtensorMap); }

// Tile geometry for R2 real rows per channel.
void tc_geometry(int R2, int Tpad, int *G, int *NG, int *boxrows, int *tmem_cols, size_t *smem)
{
	*G = 128 / R2;
	*NG = 2;
	int br = (*NG - 1) * (*G) * R2 + 128;
	if(br > 256)
	{
		*NG = 1;
		br = 128;
	}
	*boxrows = br;
	*tmem_cols = *NG == 2 ? 256 : 128;
	const size_t stage = ((size_t)br * kRowBytes + 1023) & ~(size_t)1023;
	*smem = stage * kStages + 1024;
	(void)Tpad;
}

void launch_xmac_tc(const void *tmap, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf, int nchan,
                    const int64_t *rowbase, int Tpad, int R2, int32_t *err, float2 *acc, cudaStream_t stream)
{
	int G, NG, boxrows, cols;
	size_t smem;
	tc_geometry(R2, Tpad, &G, &NG, &boxrows, &cols, &smem);
	TcParams tp;
	tp.Tpad = Tpad;
	tp.R2 = R2;
	tp.G = G;
	tp.NG = NG;
	tp.boxrows = boxrows;
	tp.tmem_cols = cols;
	tp.err = err;
	if(((uintptr_t)tmap & 63) != 0)
		return;                      // refused by tc_make_tensormap at set-up already
	cudaFuncSetAttribute(k_xmac_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	const int per = G * NG;
	dim3 grid((nchan + per - 1) / per, nf);
	k_xmac_tc<<<grid, 128, smem, stream>>>(*(const CUtensorMap *)tmap, dplans, plan_idx, rowbase, tp, acc);
}

// bf16x2 spectra [t][row][chan] -> K-major bf16 [chan][2 row + part][Tpad]
// starting at row rowbase[f] of the K-major buffer (32 x 32 tiles through
// shared memory: coalesced along channels on the read, along time on the write)
__global__ void k_spec_kmajor(const DevFreqPlan *__restrict__ plans, const int32_t *__restrict__ idx, int nrow,
                              int nchan, int T, int Tpad, const int64_t *__restrict__ rowbase,
                              const uint32_t *__restrict__ specn, uint16_t *__restrict__ kmaj)
{
	__shared__ uint32_t tile[32][33];
	const int f = idx[blockIdx.z / nrow];
	const int row = blockIdx.z % nrow;
	const int64_t spec_off = plans[f].spec_off;
	const int r2pad = plans[f].r2pad;
	const int c0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
	for(int i = threadIdx.y; i < 32; i += blockDim.y)
	{
		const int t = t0 + i, c = c0 + threadIdx.x;
		tile[i][threadIdx.x] = (t < T && c < nchan) ? specn[spec_off + ((int64_t)t * nrow + row) * nchan + c] : 0u;
	}
	__syncthreads();
	for(int i = threadIdx.y; i < 32; i += blockDim.y)
	{
		const int c = c0 + i, t = t0 + threadIdx.x;
		if(c < nchan && t < T)
		{
			const uint32_t v = tile[threadIdx.x][i];
			const int64_t base = (rowbase[f] + (int64_t)c * r2pad + 2 * row) * Tpad + t;
			kmaj[base] = (uint16_t)(v & 0xFFFFu);
			kmaj[base + Tpad] = (uint16_t)(v >> 16);
		}
	}
}

void launch_spec_kmajor(const DevFreqPlan *dplans, const int32_t *plan_idx, int nf, int nrow, int nchan, int T,
                        int Tpad, const int64_t *rowbase, const uint32_t *specn, uint16_t *kmaj, cudaStream_t stream)
{
	if(nf <= 0 || nrow <= 0)
		return;
	dim3 grid((nchan + 31) / 32, (T + 31) / 32, nf * nrow);
	k_spec_kmajor<<<grid, dim3(32, 8), 0, stream>>>(dplans, plan_idx, nrow, nchan, T, Tpad, rowbase, specn, kmaj);
}

}  // namespace fxb
