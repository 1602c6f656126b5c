// Tensor-core cross-multiply-accumulate for sm_100a (tcgen05 + TMA).
//
// Core::processdata's XMAC (mpifxcorr/src/core.cpp:877-972) and the Mode
// autocorrelations (mode.cpp:1293-1369) per channel are V = X X^H, with X the
// [inputs x time] matrix of one channel's spectra.  With A = X written as real
// rows (2 rows per input: real and imaginary part, interleaved), A A^T holds
// every product: for inputs a, b
//     Re V[a][b] = P[2a][2b] + P[2a+1][2b+1],  Im V[a][b] = P[2a+1][2b] - P[2a][2b+1].
//
// FP8 form: the same, with the spectra quantised to e4m3 pairs (one 16-bit
// word per complex value) with a scale per (channel, input) by k_quant_fp8,
// K tiles of 64 times (still 64-byte operand rows), kind::f8f6f4 MMAs of
// K = 32, and the epilogue dividing each product by the two inputs' scales.
//
// Input: the F stage's half2 (or bf16x2) spectra X 2^-kTcSpecExp, per group of
// equally shaped subbands
// one block [subband][Tpad][block][nrow][CB] (times T..Tpad-1 zero), with CB
// the channels of one work unit.  A unit is two M = 128 operand tiles of
// G = floor(128 / R2p) channels each, R2p the real rows per channel rounded up
// to 8 (rows past G R2p stay zero).  One tcgen05.mma (kind::f16, M = N = 128,
// K = 16) uses the same shared-memory tile as A and B, so the G diagonal
// R2p x R2p blocks of each 128 x 128 FP32 accumulator are the G channels'
// A A^T.  FP16 operands (11-bit significands) are the default; BF16 (8 bits)
// is kept as a measured alternative.  The epilogue multiplies every product
// by 2^(2 kTcSpecExp), which undoes the spectra's scale exactly.  A unit's two accumulators take 256 tensor-memory columns; two units
// alternate, so the epilogue of one overlaps the MMAs of the next.
//
// One persistent CTA per SM, warp-specialised:
//   warp 0     TMA producer: 3D boxes {nrow * CB values, 1 block, 32 times}
//              (each of the 32 rows one contiguous run; no multicast) into a
//              ring of raw stages,
//   warp 1     tensor-memory owner and MMA issuer,
//   warps 2-5  transposers: raw boxes -> K-major operand tiles with 64-byte
//              swizzle (a ring of operand stages),
//   warps 6-9  epilogue: copy the unit's accumulator rows of its channels to
//              shared memory and release the tensor memory at once, then form
//              every output V[a][b] from its four real products and add it
//              to the [channel][output] accumulators with vector reductions.
// Every wait is bounded: on timeout the CTA records an error code, drains its
// TMA loads and MMAs, and still releases its tensor memory.

#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cstring>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

namespace {

constexpr int kKT = 32;                    // times per K tile (64 bytes of BF16 per operand row)
constexpr int kKT8 = 64;                   // FP8 form: times per K tile (64 bytes of e4m3 per operand row)
constexpr int kRS = 6;                     // raw stages at most (tc_shape picks how many fit)
constexpr int kAS = 4;                     // operand stages at most
constexpr int kNG = 2;                     // M tiles per work unit
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

__device__ __forceinline__ void mma_f8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate)
{
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
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

// FP8 form: from four consecutive times' words of two neighbouring values
// (bytes: value 0 re, im, value 1 re, im), the four real bytes and the four
// imaginary bytes of one value in time order; sel 0x5140 picks value 0,
// 0x7362 value 1
__device__ __forceinline__ void split4(const uint32_t *w, uint32_t sel, uint32_t &re, uint32_t &im)
{
	const uint32_t p01 = __byte_perm(w[0], w[1], sel), p23 = __byte_perm(w[2], w[3], sel);
	re = __byte_perm(p01, p23, 0x5410);
	im = __byte_perm(p01, p23, 0x7632);
}

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

// the launch's common shape (every group has the same rows); the groups'
// own extents are in XMultiArgs
struct TcParams {
	int32_t nrow, r2p, G, CB;       // inputs, real rows per channel (padded to 8), channels per tile, per unit
	int32_t raw_bytes, raw_stride;  // bytes per raw box, stage stride
	int32_t nrs, nas;               // raw and operand stages in use
	int32_t dstride, dump_off;      // floats per row of the accumulator copy, its byte offset in shared memory
	int32_t rpitch;                 // values per time of one raw box (FP8 form: padded to 8)
	int32_t h16;                    // FP16 operands (else BF16)
	int32_t *err;
};

// NB: accumulator buffers per CTA.  2: 512 tensor-memory columns, the
// epilogue of one unit overlaps the MMAs of the next, one CTA per SM; 1: 256
// columns, two CTAs per SM overlap each other instead
// unit u of a launch: its group, subband of the group and channel block
struct UnitLoc {
	int gi, fi, blk;
};
__device__ __forceinline__ UnitLoc locate(const XMultiArgs &xm, int u)
{
	int gi = 0;
	while(gi + 1 < xm.ngroups && u >= xm.g[gi + 1].unit0)
		gi++;
	const int lu = u - xm.g[gi].unit0, nblk = xm.g[gi].nblk;
	const int fi = lu / nblk;
	return UnitLoc{gi, fi, lu - fi * nblk};
}

// Work units of every group of the launch in turn (a group's units are its
// subbands' channel blocks), CTAs striding over them.
template <bool F8, int NB>
__global__ void __launch_bounds__(kThreads, 3 - NB) k_xmac_tc(const __grid_constant__ XMultiArgs xm, TcParams tp)
{
	extern __shared__ __align__(1024) unsigned char smem_tc[];
	__shared__ uint64_t full_raw[kRS], empty_raw[kRS], full_a[kAS], empty_a[kAS], acc_full[NB], acc_empty[NB], mma_done;
	__shared__ uint32_t tmem_base_s;
	__shared__ volatile int fail_s;
	__shared__ int issued_s, consumed_s;

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	unsigned char *base = (unsigned char *)(((uintptr_t)smem_tc + 1023) & ~(uintptr_t)1023);
	unsigned char *raw0 = base;
	unsigned char *a0 = raw0 + (size_t)tp.nrs * tp.raw_stride;
	float *dump = (float *)(base + tp.dump_off);
	const int nrs = tp.nrs, nas = tp.nas;
	constexpr int kStageBytes = kNG * kTileBytes;

	// operand tiles start zero: rows past G R2p and padding rows are never written
	for(int i = threadIdx.x; i < nas * kStageBytes / 16; i += blockDim.x)
		((uint4 *)a0)[i] = make_uint4(0u, 0u, 0u, 0u);
	if(threadIdx.x == 0)
	{
		for(int s = 0; s < nrs; s++)
		{
			mbar_init(&full_raw[s], 1);
			mbar_init(&empty_raw[s], 4);
		}
		for(int s = 0; s < nas; s++)
		{
			mbar_init(&full_a[s], 4);
			mbar_init(&empty_a[s], 1);
		}
		for(int b = 0; b < NB; b++)
		{
			mbar_init(&acc_full[b], 1);
			mbar_init(&acc_empty[b], 4);
		}
		mbar_init(&mma_done, 1);
		fail_s = 0;
		issued_s = 0;
		consumed_s = 0;
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	if(warp == 1)
	{
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_s)),
		             "r"(256u * NB));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
	}
	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	const uint32_t tmem = tmem_base_s;
	constexpr int KT = F8 ? kKT8 : kKT;

	if(warp == 0)
	{
		if(lane == 0)
		{
			// ---- TMA producer
			int kk = 0;
			bool ok = true;
			for(int u = blockIdx.x; u < xm.nunits && ok; u += gridDim.x)
			{
				const UnitLoc L = locate(xm, u);
				const int nkt = xm.g[L.gi].nkt;
				const CUtensorMap *map = (const CUtensorMap *)&xm.map[L.gi];
				for(int kt = 0; kt < nkt; kt++, kk++)
				{
					const int s = kk % nrs;
					if(kk >= nrs && !mbar_wait(&empty_raw[s], ((kk / nrs) - 1) & 1, &fail_s))
					{
						fail_s = 1;
						ok = false;
						break;
					}
					mbar_expect_tx(&full_raw[s], (uint32_t)tp.raw_bytes);
					tma_load_3d(raw0 + (size_t)s * tp.raw_stride, map, 0, L.blk, (L.fi * nkt + kt) * KT, &full_raw[s]);
					issued_s = kk + 1;
				}
			}
		}
	}
	else if(warp == 1)
	{
		if(lane == 0)
		{
			// ---- MMA issuer: M = N = 128, FP16 x FP16 or BF16 x BF16 (FP8 form:
			// e4m3 x e4m3) -> FP32, A and B K-major; unit ku accumulates into
			// columns 256 (ku & 1).  Instruction descriptor: D format F32 (bit 4),
			// A / B formats (bits 7-9 / 10-12: 0 F16 or E4M3, 1 BF16), N >> 3
			// (bits 17-22), M >> 4 (bits 24-28).
			const uint32_t ab = (F8 || tp.h16) ? 0u : (1u << 7) | (1u << 10);
			const uint32_t idesc = (1u << 4) | ab | ((128u >> 3) << 17) | ((128u >> 4) << 24);
			int kk = 0, ku = 0;
			bool ok = true;
			for(int u = blockIdx.x; u < xm.nunits && ok; u += gridDim.x, ku++)
			{
				const int nkt = xm.g[locate(xm, u).gi].nkt;
				const int buf = ku % NB;
				if(ku >= NB)
				{
					// the epilogue has copied out this buffer's previous unit
					if(!mbar_wait(&acc_empty[buf], ((ku / NB) - 1) & 1, &fail_s))
					{
						fail_s = 3;
						ok = false;
						break;
					}
					asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
				}
				for(int kt = 0; kt < nkt; kt++, kk++)
				{
					const int s = kk % nas;
					if(!mbar_wait(&full_a[s], (kk / nas) & 1, &fail_s))
					{
						fail_s = 2;
						ok = false;
						break;
					}
					asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
					const uint32_t sbase = smem_u32(a0 + (size_t)s * kStageBytes);
#pragma unroll
					for(int g = 0; g < kNG; g++)
#pragma unroll
						for(int k2 = 0; k2 < 2; k2++)
						{
							// each MMA takes 32 bytes of every operand row (K = 16 BF16 or 32 e4m3)
							const uint64_t d = make_sdesc64(sbase + (uint32_t)(g * kTileBytes + k2 * 32));
							if constexpr(F8)
								mma_f8(tmem + (uint32_t)(buf * 256 + g * 128), d, d, idesc, (kt > 0 || k2 > 0) ? 1u : 0u);
							else
								mma_bf16(tmem + (uint32_t)(buf * 256 + g * 128), d, d, idesc,
								         (kt > 0 || k2 > 0) ? 1u : 0u);
						}
					mma_commit(&empty_a[s]);
				}
				if(ok)
					mma_commit(&acc_full[buf]);
			}
			// every MMA issued by this thread has completed once this arrives
			mma_commit(&mma_done);
			if(!mbar_wait(&mma_done, 0, &fail_s))
				fail_s = 4;
		}
	}
	else if(warp < 6)
	{
		// ---- transposers: raw [32 t][nrow][CB] bf16x2 -> operand rows.
		// Input `row` of channel cl (tile g = cl / G, slot q = cl % G) sits at
		// position p = (row + cl) mod nrow of its channel block: rows
		// m = q R2p + 2 p (real) and m + 1 (imaginary), 64-byte swizzle.  The
		// rotation by cl, and the alternating order of the two stores, spread
		// the 16-byte stores of neighbouring threads over all banks.
		const int tt = threadIdx.x - 64;
		const int rc = tp.nrow * tp.CB;                // even: CB = 2 G
		const int npairs = rc >> 1;
		const int items = 4 * npairs;                  // (8-time chunk (FP8: 16 times), pair of neighbouring values)
		constexpr int kMaxItems = 2;                   // 4 * 128 / 2 / 128
		int src_off[kMaxItems], dst_a[kMaxItems][2], dst_b[kMaxItems][2];
		uint32_t swapm[kMaxItems];
#pragma unroll
		for(int j = 0; j < kMaxItems; j++)
		{
			const int i = tt + 128 * j;
			src_off[j] = -1;
			swapm[j] = 0;
			if(i < items)
			{
				const int tc = i / npairs, pr = i - tc * npairs;
				if constexpr(F8)
					src_off[j] = tc * 16 * (tp.rpitch >> 1) + pr;  // in 4-byte units
				else
					src_off[j] = (tc * 8 * rc + 2 * pr) >> 1;      // in 8-byte units
#pragma unroll
				for(int e = 0; e < 2; e++)
				{
					const int rem = 2 * pr + e;
					const int row = rem / tp.CB, cl = rem - row * tp.CB;
					const int g = cl / tp.G, q = cl - g * tp.G;
					const int pos = (row + cl) % tp.nrow;
					const int m = q * tp.r2p + 2 * pos;
					const int sw = (tc ^ ((m >> 1) & 3)) << 4;     // rows m, m+1 share the swizzle phase
					const int re_off = g * kTileBytes + m * 64 + sw, im_off = re_off + 64;
					const bool swp = (rem >> 2) & 1;               // first store takes the imaginary row
					dst_a[j][e] = swp ? im_off : re_off;
					dst_b[j][e] = swp ? re_off : im_off;
					swapm[j] |= (uint32_t)swp << e;
				}
			}
		}
		int kk = 0;
		bool ok = true;
		for(int u = blockIdx.x; u < xm.nunits && ok; u += gridDim.x)
		{
			const int nkt = xm.g[locate(xm, u).gi].nkt;
			for(int kt = 0; kt < nkt; kt++, kk++)
			{
				const int rs = kk % nrs, as = kk % nas;
				if(!mbar_wait(&full_raw[rs], (kk / nrs) & 1, &fail_s) ||
				   (kk >= nas && !mbar_wait(&empty_a[as], ((kk / nas) - 1) & 1, &fail_s)))
				{
					fail_s = 5;
					ok = false;
					break;
				}
				const uint2 *raw = (const uint2 *)(raw0 + (size_t)rs * tp.raw_stride);
				unsigned char *A = a0 + (size_t)as * kStageBytes;
				if constexpr(F8)
				{
					const uint32_t *raw32 = (const uint32_t *)(raw0 + (size_t)rs * tp.raw_stride);
					const int tstep = tp.rpitch >> 1;
#pragma unroll
					for(int j = 0; j < kMaxItems; j++)
					{
						if(src_off[j] < 0)
							continue;
						const uint32_t *src = raw32 + src_off[j];
						uint32_t w[16];
#pragma unroll
						for(int t = 0; t < 16; t++)
							w[t] = src[t * tstep];
						uint4 re0, im0, re1, im1;
						split4(w + 0, 0x5140, re0.x, im0.x);
						split4(w + 4, 0x5140, re0.y, im0.y);
						split4(w + 8, 0x5140, re0.z, im0.z);
						split4(w + 12, 0x5140, re0.w, im0.w);
						split4(w + 0, 0x7362, re1.x, im1.x);
						split4(w + 4, 0x7362, re1.y, im1.y);
						split4(w + 8, 0x7362, re1.z, im1.z);
						split4(w + 12, 0x7362, re1.w, im1.w);
						const bool s0 = swapm[j] & 1u, s1 = (swapm[j] >> 1) & 1u;
						*(uint4 *)(A + dst_a[j][0]) = s0 ? im0 : re0;
						*(uint4 *)(A + dst_b[j][0]) = s0 ? re0 : im0;
						*(uint4 *)(A + dst_a[j][1]) = s1 ? im1 : re1;
						*(uint4 *)(A + dst_b[j][1]) = s1 ? re1 : im1;
					}
				}
				else
				{
#pragma unroll
				for(int j = 0; j < kMaxItems; j++)
				{
					if(src_off[j] < 0)
						continue;
					const uint2 *src = raw + src_off[j];
					uint2 w[8];
#pragma unroll
					for(int t = 0; t < 8; t++)
						w[t] = src[t * npairs];
					uint4 re0, im0, re1, im1;
					re0.x = __byte_perm(w[0].x, w[1].x, 0x5410);
					re0.y = __byte_perm(w[2].x, w[3].x, 0x5410);
					re0.z = __byte_perm(w[4].x, w[5].x, 0x5410);
					re0.w = __byte_perm(w[6].x, w[7].x, 0x5410);
					im0.x = __byte_perm(w[0].x, w[1].x, 0x7632);
					im0.y = __byte_perm(w[2].x, w[3].x, 0x7632);
					im0.z = __byte_perm(w[4].x, w[5].x, 0x7632);
					im0.w = __byte_perm(w[6].x, w[7].x, 0x7632);
					re1.x = __byte_perm(w[0].y, w[1].y, 0x5410);
					re1.y = __byte_perm(w[2].y, w[3].y, 0x5410);
					re1.z = __byte_perm(w[4].y, w[5].y, 0x5410);
					re1.w = __byte_perm(w[6].y, w[7].y, 0x5410);
					im1.x = __byte_perm(w[0].y, w[1].y, 0x7632);
					im1.y = __byte_perm(w[2].y, w[3].y, 0x7632);
					im1.z = __byte_perm(w[4].y, w[5].y, 0x7632);
					im1.w = __byte_perm(w[6].y, w[7].y, 0x7632);
					const bool s0 = swapm[j] & 1u, s1 = (swapm[j] >> 1) & 1u;
					*(uint4 *)(A + dst_a[j][0]) = s0 ? im0 : re0;
					*(uint4 *)(A + dst_b[j][0]) = s0 ? re0 : im0;
					*(uint4 *)(A + dst_a[j][1]) = s1 ? im1 : re1;
					*(uint4 *)(A + dst_b[j][1]) = s1 ? re1 : im1;
				}
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
		const int nin = tp.nrow, ds = tp.dstride;
		constexpr int kOB = 8;                   // outputs per thread with sources in registers
		int srcv[kOB];
		const int32_t *src_plan = nullptr;
		int src_nout = -1;
		int ku = 0;
		for(int u = blockIdx.x; u < xm.nunits; u += gridDim.x, ku++)
		{
			const int buf = ku % NB;
			const UnitLoc L = locate(xm, u);
			const XGroupRec &GR = xm.g[L.gi];
			const DevFreqPlan &P = GR.plans[GR.plan_idx[L.fi]];
			float2 *const acc = GR.acc;
			const int nout = P.acc_cstride;
			const int c_first = L.blk * tp.CB;
			const int ncv = min(tp.CB, GR.nchan - c_first);
			bool bad = !mbar_wait(&acc_full[buf], (ku / NB) & 1, &fail_s);
			if(bad)
				fail_s = 6;
			if(epi_sync_or(bad))
				break;                        // all four warps leave together
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			// 1. copy each channel's 2 nin x 2 nin block of the accumulators to
			// dump[cl][r2][c2] (rows of ds floats), then release the buffer
			for(int g = 0; g < kNG; g++)
			{
				const int qlo = (32 * lq) / tp.r2p;
				const int qhi = min(tp.G - 1, (32 * lq + 31) / tp.r2p);
				for(int q = qlo; q <= qhi; q++)
				{
					const int cl = g * tp.G + q;
					const int r2 = row - q * tp.r2p;
					const bool keep = r2 >= 0 && r2 < 2 * nin && cl < ncv;
					float *drow = dump + ((size_t)cl * 2 * nin + (keep ? r2 : 0)) * ds;
					const uint32_t tbase =
					    tmem + ((uint32_t)(32 * lq) << 16) + (uint32_t)(buf * 256 + g * 128 + q * tp.r2p);
					for(int j0 = 0; j0 < 2 * nin; j0 += 32)
					{
						float pv[32];
						const int nl = min(4, (2 * nin - j0 + 7) >> 3);
#pragma unroll
						for(int c = 0; c < 4; c++)
							if(c < nl)
								tmem_ld8(tbase + (uint32_t)(j0 + 8 * c), pv + 8 * c);
						tmem_ld_wait();
						if(keep)
						{
#pragma unroll
							for(int c = 0; c < 4; c++)
								if(c < nl)
								{
									*(float4 *)(drow + j0 + 8 * c) = make_float4(pv[8 * c], pv[8 * c + 1], pv[8 * c + 2], pv[8 * c + 3]);
									*(float4 *)(drow + j0 + 8 * c + 4) =
									    make_float4(pv[8 * c + 4], pv[8 * c + 5], pv[8 * c + 6], pv[8 * c + 7]);
								}
						}
					}
				}
			}
			asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
			__syncwarp();
			if(lane == 0)
				mbar_arrive(&acc_empty[buf]);
			epi_sync();
			// 2. outputs: V[a][b] = (P[2a][2b] + P[2a+1][2b+1], P[2a+1][2b] - P[2a][2b+1]) with
			// input a of channel cl at position (a + cl) mod nin; vector reductions
			// into the contiguous [channel][output] block (one addition per output
			// and subint, so the sum is that of a load-add-store)
			const int32_t *outsrc = P.outsrc;
			const float *isc = F8 ? P.iscale + (int64_t)c_first * nin : nullptr;   // FP8 form: [channel][input] 1 / scale
			constexpr float unscale = (float)(1 << (2 * kTcSpecExp));
			float2 *dst = acc + P.acc_off + (int64_t)c_first * nout;
			// the thread's first kOB outputs: sources held in registers (read
			// again only when the plan changes), every channel's reductions of
			// them issued back to back
			if(outsrc != src_plan || nout != src_nout)
			{
				src_plan = outsrc;
				src_nout = nout;
#pragma unroll
				for(int j = 0; j < kOB; j++)
				{
					const int o = et + 128 * j;
					srcv[j] = o < nout ? __ldg(outsrc + o) : -1;
				}
			}
			{
				int cln = 0;                      // cl mod nin
				for(int cl = 0; cl < ncv; cl++)
				{
#pragma unroll
					for(int j = 0; j < kOB; j++)
					{
						const int src = srcv[j];
						if(src < 0)
							continue;
						const int a = src & 0xFF, b = (src >> 8) & 0xFF;
						int pa = a + cln, pb = b + cln;
						if(pa >= nin)
							pa -= nin;
						if(pb >= nin)
							pb -= nin;
						const float *r0 = dump + ((size_t)cl * 2 * nin + 2 * pa) * ds + 2 * pb, *r1 = r0 + ds;
						const float2 x0 = *(const float2 *)r0, x1 = *(const float2 *)r1;
						float vre = x0.x + x1.y;
						float vim = x1.x - x0.y;
						if constexpr(F8)
						{
							const float f = isc[cl * nin + a] * isc[cl * nin + b];
							vre *= f;
							vim *= f;
						}
						else
						{
							vre *= unscale;
							vim *= unscale;
						}
						atomicAdd(dst + (int64_t)cl * nout + et + 128 * j, make_float2(vre, (src >> 16) ? -vim : vim));
					}
					if(++cln == nin)
						cln = 0;
				}
			}
			for(int o = et + 128 * kOB; o < nout; o += 128)
			{
				const int src = __ldg(outsrc + o);
				if(src < 0)
					continue;
				const int a = src & 0xFF, b = (src >> 8) & 0xFF;
				const bool cj = (src >> 16) != 0;
				int cln = 0;                      // cl mod nin
				for(int cl = 0; cl < ncv; cl++)
				{
					int pa = a + cln, pb = b + cln;
					if(pa >= nin)
						pa -= nin;
					if(pb >= nin)
						pb -= nin;
					const float *r0 = dump + ((size_t)cl * 2 * nin + 2 * pa) * ds + 2 * pb, *r1 = r0 + ds;
					float vre = r0[0] + r1[1];
					float vim = r1[0] - r0[1];
					if constexpr(F8)
					{
						const float f = isc[cl * nin + a] * isc[cl * nin + b];
						vre *= f;
						vim *= f;
					}
					else
					{
						vre *= unscale;
						vim *= unscale;
					}
					atomicAdd(dst + (int64_t)cl * nout + o, make_float2(vre, cj ? -vim : vim));
					if(++cln == nin)
						cln = 0;
				}
			}
			epi_sync();                       // the copy area is free for the next unit
		}
	}

	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	if(threadIdx.x == 0)
	{
		// on the error path, wait (bounded) for TMA loads that nobody consumed
		for(int kk = consumed_s; kk < issued_s; kk++)
			mbar_wait(&full_raw[kk % nrs], (kk / nrs) & 1, &fail_s);
		if(fail_s && tp.err)
			atomicExch(tp.err, fail_s);
	}
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	if(warp == 1)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(256u * NB));
}

// ---------------------------------------------------------------- host side
typedef CUresult (*PFN_encodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                     const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

bool tc_shape(int nrow, int nchan, int T, bool f8, bool h16, TcShape *s)
{
	s->f8 = f8 ? 1 : 0;
	s->h16 = h16 ? 1 : 0;
	s->nrow = nrow;
	s->nchan = nchan;
	s->r2p = (2 * nrow + 7) & ~7;
	if(s->r2p > 128 || nrow <= 0)
		return false;
	s->G = 128 / s->r2p;
	s->CB = kNG * s->G;
	const int kt = f8 ? kKT8 : kKT;
	s->Tpad = (T + kt - 1) / kt * kt;
	s->w8 = (nrow * s->CB + 7) & ~7;
	s->raw_bytes = f8 ? s->w8 * kKT8 * 2 : s->CB * nrow * kKT * 4;
	s->raw_stride = (s->raw_bytes + 1023) & ~1023;
	s->dstride = s->r2p + 4;
	// deepest rings that fit beside the accumulator copy
	static const int order[][2] = {{6, 4}, {6, 3}, {5, 3}, {5, 2}, {4, 2}, {3, 2}, {2, 2}};
	for(const auto &o : order)
		if(tc_stages(s, o[0], o[1]))
			return true;
	return false;
}

bool tc_stages(TcShape *s, int nrs, int nas, int nb)
{
	if(nrs < 1 || nrs > kRS || nas < 1 || nas > kAS || nb < 1 || nb > 2)
		return false;
	const size_t dump = (size_t)s->CB * 2 * s->nrow * s->dstride * 4;
	const size_t rings = (size_t)nrs * s->raw_stride + (size_t)nas * kNG * kTileBytes;
	if(1024 + rings + dump > (nb == 2 ? 227 : 112) * 1024)
		return false;
	s->nrs = nrs;
	s->nas = nas;
	s->nb = nb;
	s->dump_off = (int32_t)rings;
	s->smem = 1024 + rings + dump;
	return true;
}

// 3D map over one group's spectra [nf * Tpad][nblk][nrow * CB] of 4-byte
// bf16x2 values; box {nrow * CB, 1 block, 32 times}: each of its 32 rows is
// one contiguous run of nrow * CB <= 256 values.
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
	// FP8 form: 16-bit e4m3 pairs, rows padded to w8 values (16 bytes), 64 times
	const cuuint64_t W = s.f8 ? (cuuint64_t)s.w8 : (cuuint64_t)s.nrow * s.CB;
	const cuuint64_t esz = s.f8 ? 2 : 4;
	const cuuint64_t nblk = (cuuint64_t)((s.nchan + s.CB - 1) / s.CB);
	if(W > 256 || (W * esz) % 16 != 0)
		return false;
	cuuint64_t dims[3] = {W, nblk, (cuuint64_t)s.Tpad * nf};
	cuuint64_t strides[2] = {W * esz, nblk * W * esz};
	cuuint32_t box[3] = {(cuuint32_t)W, 1, (cuuint32_t)(s.f8 ? kKT8 : kKT)};
	cuuint32_t estr[3] = {1, 1, 1};
	CUresult r = encode((CUtensorMap *)map_out, s.f8 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT32,
	                    3, (void *)spec, dims, strides, box,
	                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
	                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	return r == CUDA_SUCCESS;
}

size_t tc_tensormap_size() { return sizeof(CUtensorMap); }

bool xmac_multi_add(XMultiArgs *xm, const void *tmap, const TcShape &s, const DevFreqPlan *dplans,
                    const int32_t *plan_idx, int nf, float2 *acc)
{
	if(xm->ngroups >= kXMultiGroups || ((uintptr_t)tmap & 63) != 0 || nf <= 0)
		return false;
	XGroupRec &g = xm->g[xm->ngroups];
	memcpy(&xm->map[xm->ngroups], tmap, sizeof(CUtensorMap));
	g.plans = dplans;
	g.plan_idx = plan_idx;
	g.acc = acc;
	g.nchan = s.nchan;
	g.nkt = s.Tpad / (s.f8 ? kKT8 : kKT);
	g.nblk = (s.nchan + s.CB - 1) / s.CB;
	g.unit0 = xm->nunits;
	xm->nunits += g.nblk * nf;
	xm->ngroups++;
	return true;
}

void launch_xmac_tc_multi(const XMultiArgs &xm, const TcShape &s, int nsm, int32_t *err, cudaStream_t stream)
{
	if(xm.ngroups <= 0 || xm.nunits <= 0)
		return;
	TcParams tp;
	tp.nrow = s.nrow;
	tp.r2p = s.r2p;
	tp.G = s.G;
	tp.CB = s.CB;
	tp.rpitch = s.f8 ? s.w8 : s.nrow * s.CB;
	tp.raw_bytes = s.raw_bytes;
	tp.raw_stride = s.raw_stride;
	tp.nrs = s.nrs;
	tp.nas = s.nas;
	tp.dstride = s.dstride;
	tp.dump_off = s.dump_off;
	tp.h16 = s.h16;
	tp.err = err;
	const int ctas = nsm * (s.nb == 1 ? 2 : 1);
	const int grid = xm.nunits < ctas ? xm.nunits : ctas;
	if(s.f8 && s.nb == 1)
	{
		cudaFuncSetAttribute(k_xmac_tc<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
		k_xmac_tc<true, 1><<<grid, kThreads, s.smem, stream>>>(xm, tp);
	}
	else if(s.f8)
	{
		cudaFuncSetAttribute(k_xmac_tc<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
		k_xmac_tc<true, 2><<<grid, kThreads, s.smem, stream>>>(xm, tp);
	}
	else if(s.nb == 1)
	{
		cudaFuncSetAttribute(k_xmac_tc<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
		k_xmac_tc<false, 1><<<grid, kThreads, s.smem, stream>>>(xm, tp);
	}
	else
	{
		cudaFuncSetAttribute(k_xmac_tc<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
		k_xmac_tc<false, 2><<<grid, kThreads, s.smem, stream>>>(xm, tp);
	}
}

void launch_xmac_tc(const void *tmap, const TcShape &s, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf,
                    int nsm, int32_t *err, float2 *acc, cudaStream_t stream)
{
	XMultiArgs xm;
	memset(&xm, 0, sizeof(xm));
	if(!xmac_multi_add(&xm, tmap, s, dplans, plan_idx, nf, acc))
		return;                      // refused by tc_make_tensormap at set-up already
	launch_xmac_tc_multi(xm, s, nsm, err, stream);
}

// ---------------------------------------------------------------- FP8 quantisation
// One CTA per (channel block, subband); thread = one (input, channel) column
// of the block.  Two passes over the subint's T times: the column's largest
// |re| or |im|, then the scaled e4m3 pairs (saturating, round to nearest).
// Columns of channels past nchan hold zeros and keep scale 1.  The source
// spectra (half2, or bf16x2) hold X 2^-kTcSpecExp; the inverse scale written
// per (channel, input) includes 2^kTcSpecExp, so that the epilogue's product
// of two inverse scales restores X X^H.
__device__ __forceinline__ float2 spec_value(uint32_t w, bool h16)
{
	if(h16)
		return __half22float2(*(const __half2 *)&w);
	return __bfloat1622float2(*(const __nv_bfloat162 *)&w);
}

__global__ void k_quant_fp8(const DevFreqPlan *__restrict__ plans, const int32_t *__restrict__ plan_idx, int T,
                            int w8, int h16, const uint32_t *__restrict__ spec16, uint16_t *__restrict__ spec8)
{
	const DevFreqPlan &P = plans[plan_idx[blockIdx.y]];
	const int blk = blockIdx.x;
	const int W = P.nrow * P.tcb;
	const int col = threadIdx.x;
	if(col >= W || blk >= P.tnblk)
		return;
	const int row = col / P.tcb, cl = col - row * P.tcb;
	const int64_t ts16 = (int64_t)P.tnblk * W, ts8 = (int64_t)P.tnblk * w8;
	const uint32_t *src = spec16 + P.spec_off + (int64_t)blk * W + col;
	float amax = 0.0f;
	for(int t = 0; t < T; t++)
	{
		const float2 v = spec_value(__ldg(src + t * ts16), h16 != 0);
		amax = fmaxf(amax, fmaxf(fabsf(v.x), fabsf(v.y)));
	}
	const float sc = amax > 0.0f ? 240.0f / amax : 1.0f;
	uint16_t *dst = spec8 + P.spec8_off + (int64_t)blk * w8 + col;
	for(int t = 0; t < T; t++)
	{
		const float2 v = spec_value(__ldg(src + t * ts16), h16 != 0);
		dst[t * ts8] = (uint16_t)__nv_cvt_float2_to_fp8x2(make_float2(v.x * sc, v.y * sc), __NV_SATFINITE, __NV_E4M3);
	}
	const int c = blk * P.tcb + cl;
	if(c < P.nchan)
		P.iscale[(int64_t)c * P.nrow + row] = (float)(1 << kTcSpecExp) / sc;
}

void launch_quant_fp8(const TcShape &s, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf, int T,
                      const uint32_t *spec16, uint16_t *spec8, cudaStream_t stream)
{
	if(nf <= 0 || T <= 0)
		return;
	const int W = s.nrow * s.CB;
	const int nblk = (s.nchan + s.CB - 1) / s.CB;
	k_quant_fp8<<<dim3(nblk, nf), (W + 31) / 32 * 32, 0, stream>>>(dplans, plan_idx, T, s.w8, s.h16, spec16, spec8);
}

}  // namespace fxb
