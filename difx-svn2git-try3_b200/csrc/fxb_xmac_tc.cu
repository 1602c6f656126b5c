// Tensor-core cross-multiply-accumulate for sm_100a (tcgen05 + TMA).
//
// Core::processdata's XMAC (mpifxcorr/src/core.cpp:877-972) and the Mode
// autocorrelations (mode.cpp:1293-1369) per channel are V = X X^H, with X the
// [inputs x time] matrix of one channel's spectra.  With A = X written as real
// rows (2 rows per input: real and imaginary part, interleaved), A A^T holds
// every product: for inputs a, b
//     Re V[a][b] = P[2a][2b] + P[2a+1][2b+1],  Im V[a][b] = P[2a+1][2b] - P[2a][2b+1].
//
// Input: the F stage's bf16x2 spectra, per group of equally shaped subbands
// one block [subband][Tpad][nrow][nchan] (times T..Tpad-1 zero).  A work unit
// is 4 G consecutive channels of one subband, G = floor(128 / R2p) with R2p
// the real rows per channel rounded up to 8: four M = 128 operand tiles of G
// channels each (the rows past G R2p stay zero).  One tcgen05.mma (kind::f16,
// M = N = 128, K = 16) uses the same shared-memory tile as A and B, so the G
// diagonal R2p x R2p blocks of each 128 x 128 FP32 accumulator are the G
// channels' A A^T; the four accumulators fill the 512 columns of tensor memory.
//
// One persistent CTA per SM, warp-specialised:
//   warp 0     TMA producer: 3D boxes {4G channels, nrow, 32 times} of the
//              spectra (no multicast) into a 3-stage ring,
//   warp 1     tensor-memory owner and MMA issuer,
//   warps 2-5  transposers: raw boxes -> K-major operand tiles with 64-byte
//              swizzle (2-stage ring),
//   warps 6-9  epilogue: tcgen05.ld of each accumulator (released tile by tile
//              so that the next unit's MMAs start while the rest drain),
//              recombination into complex products, coalesced accumulation
//              into the [channel][output] accumulators.
// Every wait is bounded: on timeout the CTA records an error code, drains its
// TMA loads and MMAs, and still releases its tensor memory.

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

namespace {

constexpr int kKT = 32;                    // times per K tile (64 bytes of BF16 per operand row)
constexpr int kRS = 3;                     // raw stages
constexpr int kAS = 2;                     // operand stages
constexpr int kNG = 4;                     // M tiles per work unit
constexpr int kTileBytes = 128 * kKT * 2;  // one operand tile: 128 rows x 64 bytes
constexpr int kThreads = 320;
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

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// bounded wait for the phase with parity `parity`; gives up early once
// another role has recorded a failure
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *fail)
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
		if((it & 255u) == 255u && *fail)
			return false;
	}
	return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
	asm volatile(
	    "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
	        smem_u32(dst)),
	    "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
	    : "memory");
}

// shared-memory matrix descriptor: K-major, 64-byte swizzle (rows of 64
// bytes, 8-row groups 512 bytes apart), descriptor version 1 (tcgen05)
__device__ __forceinline__ uint64_t make_sdesc64(uint32_t saddr)
{
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3FFF);            // start address
	d |= (uint64_t)1 << 16;                             // leading byte offset (unused for swizzled K-major)
	d |= (uint64_t)(512 >> 4) << 32;                    // stride byte offset
	d |= (uint64_t)1 << 46;                             // descriptor version
	d |= (uint64_t)4 << 61;                             // SWIZZLE_64B
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

// named barrier of the four epilogue warps
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;\n" ::: "memory"); }

// the same barrier, returning whether any of the 128 threads passed true
__device__ __forceinline__ bool epi_sync_or(bool v)
{
	uint32_t r;
	asm volatile(
	    "{\n\t.reg .pred p, q;\n\t"
	    "setp.ne.u32 p, %1, 0;\n\t"
	    "barrier.red.or.pred q, 1, 128, p;\n\t"
	    "selp.u32 %0, 1, 0, q;\n\t}\n"
	    : "=r"(r)
	    : "r"((uint32_t)v)
	    : "memory");
	return r != 0;
}

}  // namespace

struct TcParams {
	int32_t nrow, r2p, G, CB;       // inputs, real rows per channel (padded to 8), channels per tile, per unit
	int32_t nchan, Tpad, nkt, nf;   // channels, padded times, K tiles, subbands in the group
	int32_t nblk, nunits;           // channel blocks per subband, work units
	int32_t raw_bytes, raw_stride;  // bytes per raw box, stage stride
	int32_t vbuf_floats;            // epilogue buffer capacity (floats)
	int32_t *err;
};

__global__ void __launch_bounds__(kThreads, 1) k_xmac_tc(const __grid_constant__ CUtensorMap tmap,
                                                         const DevFreqPlan *__restrict__ plans,
                                                         const int32_t *__restrict__ plan_idx, TcParams tp,
                                                         float2 *__restrict__ acc)
{
	extern __shared__ __align__(1024) unsigned char smem_tc[];
	__shared__ uint64_t full_raw[kRS], empty_raw[kRS], full_a[kAS], empty_a[kAS], acc_full, acc_empty[kNG], mma_done;
	__shared__ uint32_t tmem_base_s;
	__shared__ volatile int fail_s;
	__shared__ int issued_s, consumed_s;

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	unsigned char *base = (unsigned char *)(((uintptr_t)smem_tc + 1023) & ~(uintptr_t)1023);
	unsigned char *raw0 = base;
	unsigned char *a0 = raw0 + (size_t)kRS * tp.raw_stride;
	float2 *vbuf = (float2 *)(a0 + (size_t)kAS * kNG * kTileBytes);

	// operand tiles start zero: rows past G R2p and padding rows are never written
	for(int i = threadIdx.x; i < kAS * kNG * kTileBytes / 16; i += blockDim.x)
		((uint4 *)a0)[i] = make_uint4(0u, 0u, 0u, 0u);
	if(threadIdx.x == 0)
	{
		for(int s = 0; s < kRS; s++)
		{
			mbar_init(&full_raw[s], 1);
			mbar_init(&empty_raw[s], 4);
		}
		for(int s = 0; s < kAS; s++)
		{
			mbar_init(&full_a[s], 4);
			mbar_init(&empty_a[s], 1);
		}
		mbar_init(&acc_full, 1);
		for(int g = 0; g < kNG; g++)
			mbar_init(&acc_empty[g], 4);
		mbar_init(&mma_done, 1);
		fail_s = 0;
		issued_s = 0;
		consumed_s = 0;
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	if(warp == 1)
	{
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_s)),
		             "r"(512u));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
	}
	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	const uint32_t tmem = tmem_base_s;
	const int nkt = tp.nkt;

	if(warp == 0)
	{
		if(lane == 0)
		{
			// ---- TMA producer
			int kk = 0;
			bool ok = true;
			for(int u = blockIdx.x; u < tp.nunits && ok; u += gridDim.x)
			{
				const int fi = u / tp.nblk, blk = u - fi * tp.nblk;
				for(int kt = 0; kt < nkt; kt++, kk++)
				{
					const int s = kk % kRS;
					if(kk >= kRS && !mbar_wait(&empty_raw[s], ((kk / kRS) - 1) & 1, &fail_s))
					{
						fail_s = 1;
						ok = false;
						break;
					}
					mbar_expect_tx(&full_raw[s], (uint32_t)tp.raw_bytes);
					tma_load_3d(raw0 + (size_t)s * tp.raw_stride, &tmap, blk * tp.CB, 0, fi * tp.Tpad + kt * kKT,
					            &full_raw[s]);
					issued_s = kk + 1;
				}
			}
		}
	}
	else if(warp == 1)
	{
		if(lane == 0)
		{
			// ---- MMA issuer: M = N = 128, BF16 x BF16 -> FP32, A and B K-major
			const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
			int kk = 0, ku = 0;
			bool ok = true;
			for(int u = blockIdx.x; u < tp.nunits && ok; u += gridDim.x, ku++)
			{
				for(int kt = 0; kt < nkt && ok; kt++, kk++)
				{
					const int s = kk % kAS;
					if(!mbar_wait(&full_a[s], (kk / kAS) & 1, &fail_s))
					{
						fail_s = 2;
						ok = false;
						break;
					}
					asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
					const uint32_t sbase = smem_u32(a0 + (size_t)s * kNG * kTileBytes);
					for(int g = 0; g < kNG; g++)
					{
						if(kt == 0 && ku > 0)
						{
							// the epilogue has read this accumulator of the previous unit
							if(!mbar_wait(&acc_empty[g], (ku - 1) & 1, &fail_s))
							{
								fail_s = 3;
								ok = false;
								break;
							}
							asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
						}
#pragma unroll
						for(int k2 = 0; k2 < kKT / 16; k2++)
						{
							const uint64_t d = make_sdesc64(sbase + (uint32_t)(g * kTileBytes + k2 * 32));
							mma_bf16(tmem + (uint32_t)(g * 128), d, d, idesc, (kt > 0 || k2 > 0) ? 1u : 0u);
						}
					}
					mma_commit(&empty_a[s]);
				}
				if(ok)
					mma_commit(&acc_full);
			}
			// every MMA issued by this thread has completed once this arrives
			mma_commit(&mma_done);
			if(!mbar_wait(&mma_done, 0, &fail_s))
				fail_s = 4;
		}
	}
	else if(warp < 6)
	{
		// ---- transposers: raw [32 t][nrow][CB] bf16x2 -> operand rows
		// m = q R2p + 2 row + part of tile g (channel g G + q), 64-byte swizzle
		const int tt = threadIdx.x - 64;
		const int rc = tp.nrow * tp.CB;
		const int items = 4 * rc;
		int kk = 0;
		bool ok = true;
		for(int u = blockIdx.x; u < tp.nunits && ok; u += gridDim.x)
		{
			for(int kt = 0; kt < nkt; kt++, kk++)
			{
				const int rs = kk % kRS, as = kk % kAS;
				if(!mbar_wait(&full_raw[rs], (kk / kRS) & 1, &fail_s) ||
				   (kk >= kAS && !mbar_wait(&empty_a[as], ((kk / kAS) - 1) & 1, &fail_s)))
				{
					fail_s = 5;
					ok = false;
					break;
				}
				const uint32_t *raw = (const uint32_t *)(raw0 + (size_t)rs * tp.raw_stride);
				unsigned char *A = a0 + (size_t)as * kNG * kTileBytes;
				for(int i = tt; i < items; i += 128)
				{
					const int tc = i / rc, rem = i - tc * rc;
					const int row = rem / tp.CB, cl = rem - row * tp.CB;
					const int g = cl / tp.G, q = cl - g * tp.G;
					uint32_t w[8];
#pragma unroll
					for(int j = 0; j < 8; j++)
						w[j] = raw[(tc * 8 + j) * rc + rem];
					uint4 re, im;
					re.x = __byte_perm(w[0], w[1], 0x5410);
					re.y = __byte_perm(w[2], w[3], 0x5410);
					re.z = __byte_perm(w[4], w[5], 0x5410);
					re.w = __byte_perm(w[6], w[7], 0x5410);
					im.x = __byte_perm(w[0], w[1], 0x7632);
					im.y = __byte_perm(w[2], w[3], 0x7632);
					im.z = __byte_perm(w[4], w[5], 0x7632);
					im.w = __byte_perm(w[6], w[7], 0x7632);
					const int m = q * tp.r2p + 2 * row;
					const int sw = (tc ^ ((m >> 1) & 3)) << 4;     // rows m, m+1 share the swizzle phase
					unsigned char *tile = A + g * kTileBytes;
					*(uint4 *)(tile + m * 64 + sw) = re;
					*(uint4 *)(tile + (m + 1) * 64 + sw) = im;
				}
				// generic-proxy writes -> visible to the tensor core's async proxy
				asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
				__syncwarp();
				if(lane == 0)
				{
					mbar_arrive(&empty_raw[rs]);
					mbar_arrive(&full_a[as]);
				}
				if(tt == 0)
					consumed_s = kk + 1;
			}
		}
	}
	else
	{
		// ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31
		const int lq = warp & 3;
		const int et = threadIdx.x - 192;
		const int row = 32 * lq + lane;          // accumulator row of this thread
		int ku = 0;
		for(int u = blockIdx.x; u < tp.nunits; u += gridDim.x, ku++)
		{
			const int fi = u / tp.nblk, blk = u - fi * tp.nblk;
			const DevFreqPlan &P = plans[plan_idx[fi]];
			const int nout = P.acc_cstride;
			const int c_first = blk * tp.CB;
			for(int i = et; i < tp.CB * nout; i += 128)
				vbuf[i] = make_float2(0.0f, 0.0f);
			bool bad = !mbar_wait(&acc_full, ku & 1, &fail_s);
			if(bad)
				fail_s = 6;
			if(epi_sync_or(bad))
				break;                        // all four warps leave together
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			const int nin = tp.nrow;
			for(int g = 0; g < kNG; g++)
			{
				const int qlo = (32 * lq) / tp.r2p;
				const int qhi = min(tp.G - 1, (32 * lq + 31) / tp.r2p);
				for(int q = qlo; q <= qhi; q++)
				{
					const int cl = g * tp.G + q;
					const int r2 = row - q * tp.r2p;
					const bool mine = r2 >= 0 && r2 < 2 * nin && (r2 & 1) == 0 && c_first + cl < tp.nchan;
					const int a = r2 >> 1;
					for(int j8 = 0; j8 < 2 * nin; j8 += 8)
					{
						float pv[8];
						tmem_ld8(tmem + ((uint32_t)(32 * lq) << 16) + (uint32_t)(g * 128 + q * tp.r2p + j8), pv);
						tmem_ld_wait();
#pragma unroll
						for(int h = 0; h < 4; h++)
						{
							const int b = (j8 >> 1) + h;
							const float p_re = pv[2 * h], p_im = pv[2 * h + 1];         // P[row][2b], P[row][2b+1]
							const float o_re = __shfl_xor_sync(0xffffffffu, p_re, 1);   // partner row's P[.][2b]
							const float o_im = __shfl_xor_sync(0xffffffffu, p_im, 1);   // partner row's P[.][2b+1]
							if(!mine || b >= nin || b < a)
								continue;
							const float vre = p_re + o_im;      // P[2a][2b] + P[2a+1][2b+1]
							const float vim = o_re - p_im;      // P[2a+1][2b] - P[2a][2b+1]
							const int dA = P.destA[a * nin + b];
							const int dB = P.destB[a * nin + b];
							if(dA >= 0)
								vbuf[cl * nout + dA] = make_float2(vre, vim);
							if(dB >= 0)
								vbuf[cl * nout + dB] = make_float2(vre, -vim);
						}
					}
				}
				// this warp is done with accumulator g
				asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
				__syncwarp();
				if(lane == 0)
					mbar_arrive(&acc_empty[g]);
			}
			epi_sync();
			// coalesced accumulate into the contiguous [channel][output] block
			const int nvalid = min(tp.CB, tp.nchan - c_first) * nout;
			float2 *dst = acc + P.acc_off + (int64_t)c_first * nout;
			for(int i = et; i < nvalid; i += 128)
			{
				const float2 v = vbuf[i], o = dst[i];
				dst[i] = make_float2(o.x + v.x, o.y + v.y);
			}
			epi_sync();
		}
	}

	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	if(threadIdx.x == 0)
	{
		// on the error path, wait (bounded) for TMA loads that nobody consumed
		for(int kk = consumed_s; kk < issued_s; kk++)
			mbar_wait(&full_raw[kk % kRS], (kk / kRS) & 1, &fail_s);
		if(fail_s && tp.err)
			atomicExch(tp.err, fail_s);
	}
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	if(warp == 1)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512u));
}

// ---------------------------------------------------------------- host side
typedef CUresult (*PFN_encodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                     const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

bool tc_shape(int nrow, int nchan, int T, int nout_max, TcShape *s)
{
	s->nrow = nrow;
	s->nchan = nchan;
	s->r2p = (2 * nrow + 7) & ~7;
	if(s->r2p > 128 || nrow <= 0)
		return false;
	s->G = 128 / s->r2p;
	s->CB = kNG * s->G;
	s->Tpad = (T + kKT - 1) / kKT * kKT;
	s->raw_bytes = s->CB * nrow * kKT * 4;
	s->raw_stride = (s->raw_bytes + 1023) & ~1023;
	s->vbuf_floats = 2 * s->CB * nout_max;
	s->smem = 1024 + (size_t)kRS * s->raw_stride + (size_t)kAS * kNG * kTileBytes + (size_t)s->vbuf_floats * 4;
	return s->smem <= 227 * 1024;
}

// 3D map over one group's spectra [nf * Tpad][nrow][nchan] of 4-byte bf16x2
// values; box {CB channels, nrow, 32 times}.  The x coordinate (first
// channel of a unit) is a multiple of CB = 4 G, i.e. of 16 bytes.
bool tc_make_tensormap(void *map_out, const void *spec, const TcShape &s, int nf)
{
	if(((uintptr_t)map_out & 63) != 0 || ((uintptr_t)spec & 15) != 0)
		return false;
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
	cuuint64_t dims[3] = {(cuuint64_t)s.nchan, (cuuint64_t)s.nrow, (cuuint64_t)s.Tpad * nf};
	cuuint64_t strides[2] = {(cuuint64_t)s.nchan * 4, (cuuint64_t)s.nrow * s.nchan * 4};
	cuuint32_t box[3] = {(cuuint32_t)s.CB, (cuuint32_t)s.nrow, (cuuint32_t)kKT};
	cuuint32_t estr[3] = {1, 1, 1};
	CUresult r = encode((CUtensorMap *)map_out, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, (void *)spec, dims, strides, box,
	                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
	                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	return r == CUDA_SUCCESS;
}

size_t tc_tensormap_size() { return sizeof(CUtensorMap); }

void launch_xmac_tc(const void *tmap, const TcShape &s, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf,
                    int nsm, int32_t *err, float2 *acc, cudaStream_t stream)
{
	if(((uintptr_t)tmap & 63) != 0 || nf <= 0)
		return;                      // refused by tc_make_tensormap at set-up already
	TcParams tp;
	tp.nrow = s.nrow;
	tp.r2p = s.r2p;
	tp.G = s.G;
	tp.CB = s.CB;
	tp.nchan = s.nchan;
	tp.Tpad = s.Tpad;
	tp.nkt = s.Tpad / kKT;
	tp.nf = nf;
	tp.nblk = (s.nchan + s.CB - 1) / s.CB;
	tp.nunits = tp.nblk * nf;
	tp.raw_bytes = s.raw_bytes;
	tp.raw_stride = s.raw_stride;
	tp.vbuf_floats = s.vbuf_floats;
	tp.err = err;
	cudaFuncSetAttribute(k_xmac_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
	const int grid = tp.nunits < nsm ? tp.nunits : nsm;
	k_xmac_tc<<<grid, kThreads, s.smem, stream>>>(*(const CUtensorMap *)tmap, dplans, plan_idx, tp, acc);
}

}  // namespace fxb
