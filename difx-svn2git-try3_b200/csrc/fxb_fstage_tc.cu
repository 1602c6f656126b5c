// F stage of the tensor-core form with the FFT on the tensor cores (sm_100a).
//
// Mode::process (mpifxcorr/src/mode.cpp:845-1308) per FFT of N = 2048 points:
// decode, fringe rotation, complex FFT, sideband selection, fractional-sample
// rotation.  The FFT runs as the four-step factorisation N = 64 x 32
// (n = 32 n1 + n2, k = k1 + 64 k2):
//   Y[k1][n2] = sum_n1 F64[k1][n1] x[32 n1 + n2]         (MMA 1)
//   Y[k1][n2] *= w_N^(n2 k1)                              (CUDA cores)
//   X[k1 + 64 k2] = sum_n2 Y[k1][n2] F32[n2][k2]          (MMA 2, 16 values of k2)
// with complex products written as real ones:
//   MMA 1: rows (k1, re|im) of [[Fr, -Fi], [Fi, Fr]] (M = 128, K = 128 = (re|im, n1))
//          times columns (FFT, n2) holding (x_re[n1], x_im[n1]) (N = 128: 4 FFTs);
//   MMA 2: rows (FFT, k1) holding (Y_re[n2], Y_im[n2]) (M = 128: 2 FFTs, K = 64)
//          times columns (re|im, k2) of [[Fr, Fi], [-Fi, Fr]] (N = 32).
// Operands are FP16 (11-bit significands) with FP32 accumulation in tensor
// memory: |x| <= 38.8 (8-bit levels), so every FP16 value stays in range.
//
// A work unit is one subband of one station (its one or two polarisation
// bands) at two consecutive FFT times: 4 FFTs.  CTAs are persistent (two per
// SM); per unit the 256 threads
//   1. decode: thread (time, n1 quarter, n2) issues the loads of its 16 VDIF
//      words x[32 n1 + n2] (both bands share a word), then forms the fringe-
//      rotated samples (rotator advanced by the per-FFT step exp(-2 pi i 32 a))
//      and stores them as FP16 into the K-major operand tile,
//   2. one thread issues MMA 1 (8 x K = 16), all wait on its mbarrier,
//   3. twiddle: each thread reads its accumulator row (k1, re|im), combines it
//      with the neighbouring lane's (the other part), multiplies by the
//      twiddle and stores FP16 rows (FFT, k1) over the spent operand tile,
//   4. one thread issues MMA 2 (2 tiles x 4 x K = 16), all wait,
//   5. output: each thread reads row (FFT, k1) = 16 channels c = k1 + 64 j,
//      applies exp(+2 pi i f_c fse) (advanced by exp(2 pi i 64 dfs)) and stores
//      bf16x2 into the blocked spectra [t][block][row][tcb].
// Every wait is bounded; a timeout sets the error flag, the CTA waits
// (bounded) for its MMAs and still frees its tensor memory.

#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <vector>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

namespace {

constexpr int kN = 2048, kN1 = 64, kN2 = 32;
constexpr int kThreadsF = 256;
constexpr int kTileB = 2 * 128 * 128;          // MMA 1 operand: 2 K blocks x 128 columns x 128 bytes
constexpr int kA1 = 2 * 128 * 128;             // DFT-64 matrix: 2 K blocks x 128 rows x 128 bytes
constexpr int kB3 = 32 * 128;                  // DFT-32 columns of one sideband
constexpr uint32_t kWaitLimitF = 1u << 22;

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait_f(uint64_t *bar, uint32_t parity)
{
	const uint32_t a = su32(bar);
	for(uint32_t it = 0; it < kWaitLimitF; it++)
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

// K-major, 128-byte swizzle (8-row groups 1024 bytes apart), tcgen05 version
__device__ __forceinline__ uint64_t sdesc128(uint32_t saddr)
{
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3FFF);
	d |= (uint64_t)1 << 16;
	d |= (uint64_t)(1024 >> 4) << 32;
	d |= (uint64_t)1 << 46;
	d |= (uint64_t)2 << 61;
	return d;
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate)
{
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
	    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit_to(uint64_t *bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(su32(bar))
	             : "memory");
}

__device__ __forceinline__ void tld32(uint32_t taddr, float *v)
{
	uint32_t r[32];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
	    "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
	      "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
	      "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
	    : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
	for(int i = 0; i < 32; i++)
		v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b)
{
	const __half2 h = __floats2half2_rn(a, b);
	return *(const uint32_t *)&h;
}

// byte offset of 16-byte chunk `chunk` of row `row` in a K-major SW128 tile
__device__ __forceinline__ int swz(int row, int chunk) { return row * 128 + ((chunk ^ (row & 7)) << 4); }

__device__ __forceinline__ float level2f(uint32_t code)
{
	const float mag = ((code ^ (code >> 1)) & 1u) ? 1.0f : 3.3359f;
	return (code & 2u) ? mag : -mag;
}

__device__ __forceinline__ float fracc(double x) { return (float)(x - rint(x)); }

// constants of one FFT time of the unit
struct TcFftConst {
	float c0r, c0i;          // unused padding for alignment
	float P0, alpha;         // fringe phase (turns): start, per sample
	float Ur, Ui;            // rotator step over 32 samples: exp(-2 pi i 32 alpha)
	float dfs, postf;        // fractional-sample turns per channel, order-0 post-F turns
	float Rr, Ri;            // fractional-sample step over 64 channels: exp(2 pi i 64 dfs)
	uint32_t fa, so, fmask;
	int32_t stuck, flags;    // flags: 1 valid FFT, 2 fmask covers the window
	int32_t t;
};

}  // namespace


// Shared-memory layout (bytes from a 1024-aligned base): DFT-64 matrix,
// DFT-32 columns (upper, lower sideband), twiddles [n2][k1] (float2), the
// operand tile of MMA 1 (reused for the operand tiles of MMA 2), and the
// staging of the next unit's VDIF words ([sample][thread]).
constexpr int kOffB3 = kA1, kOffTw = kA1 + 2 * kB3, kOffB = kOffTw + kN2 * kN1 * 8;
constexpr int kOffStage = kOffB + kTileB;
constexpr int kTablesBytes = kOffB;                 // copied from the table in global memory
constexpr size_t kSmemTc = 1024 + (size_t)kOffStage + 16 * kThreadsF * 4;

namespace {

// fields of one work unit (subband of one station, two FFT times)
struct TcUnit {
	const uint8_t *buf;
	uint32_t fs, bpt, boff0, boff1;
	int nbits, header, framebytes, station, freq, row0, row1, t0;
	bool lsb, oneword, pair4;
	double lo, bw;
};

__device__ __forceinline__ TcUnit tc_unit(const FsArgs &a, int u, int count)
{
	TcUnit U;
	const FGroup &g = a.groups[a.first + u % count];     // work items fastest: a subband's stations together
	const DevStation *Sp = a.st + g.station;
	U.station = g.station;
	U.freq = g.freq;
	U.row0 = g.row[0];
	U.row1 = g.row[1];
	U.lsb = g.lsb != 0;
	U.lo = g.lofreq;
	U.fs = (uint32_t)Sp->framesamples;
	U.nbits = Sp->nbits;
	U.bpt = (uint32_t)(Sp->nband * U.nbits);
	U.header = Sp->header;
	U.framebytes = Sp->framebytes;
	U.bw = Sp->bw;
	U.buf = a.sub[g.station].buf;
	U.boff0 = (uint32_t)(g.band[0] * U.nbits);
	U.boff1 = (uint32_t)(g.band[1] * U.nbits);
	U.oneword = U.bpt <= 32;
	U.pair4 = U.nbits == 2 && U.oneword && U.boff1 == U.boff0 + 2;
	U.t0 = (u / count) * 2;
	return U;
}

// constants of FFT time t of a unit from its FFT parameters (mode.cpp:906-1097)
__device__ __forceinline__ TcFftConst tc_consts(const TcUnit &U, const FftParam &p, int t, int T, int order,
                                               int fraclo)
{
	constexpr int nchan = kN / 2;
	TcFftConst c;
	memset(&c, 0, sizeof(c));
	c.Ur = 1.0f;
	c.Rr = 1.0f;
	c.t = t;
	if(t >= T || p.status != kFftOk)
		return c;
	c.flags = 1 | (p.mflags ? 2 : 0);
	c.fmask = p.fmask;
	const uint32_t g0 = (uint32_t)p.nearest;
	c.fa = g0 / U.fs;
	c.so = g0 - c.fa * U.fs;
	c.stuck = p.stuck;
	const int idl = p.integerdelay;
	const double fl = fraclo ? (U.lo - (int)U.lo) * (double)idl : 0.0;
	if(order == 1)
	{
		c.P0 = fracc(U.lo * p.b + fl);
		c.alpha = (float)(U.lo * p.a * (1.0 / kN));
		const double step = U.lo * p.a * (32.0 / kN);
		float sn, cs;
		sincospif((float)(-2.0 * (step - rint(step))), &sn, &cs);
		c.Ur = cs;
		c.Ui = sn;
	}
	c.dfs = (float)(U.bw * (1.0 / nchan) * (double)p.fse);
	if(order == 0)
	{
		double pr = (p.averagedelay - idl) * U.lo;
		if(fraclo)
			pr += idl * (U.lo - (int)U.lo);
		c.postf = -(float)(pr - (int)pr);
	}
	const double r64 = U.bw * (64.0 / nchan) * (double)p.fse;
	float sn, cs;
	sincospif((float)(2.0 * (r64 - rint(r64))), &sn, &cs);
	c.Rr = cs;
	c.Ri = sn;
	return c;
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src, uint32_t bytes)
{
	asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

// Issue the loads of this thread's 16 VDIF words x[32 n1 + n2] of a unit
// (n1 in the warp's quarter, times by warp half) into the staging; invalid
// samples are zero-filled without a load.  Returns the valid-sample bits.
__device__ __forceinline__ uint32_t tc_prefetch(const FsArgs &a, const TcUnit &U, const TcFftConst &c, uint32_t stage_addr,
                                                int warp, int lane, int tid)
{
	const int q4 = warp & 3, n2 = lane;
	const bool active = (c.flags & 1) != 0, narrow = (c.flags & 2) != 0;
	const uint8_t *vrow = a.valid + (int64_t)U.station * a.valid_stride;
	const int nfirst = n2 + 32 * 16 * q4;
	const uint32_t xs = c.so + (uint32_t)nfirst;
	uint32_t kf = xs / U.fs, tin = xs - kf * U.fs;
	const uint8_t *fp = U.buf + ((int64_t)c.fa + kf) * U.framebytes + U.header;
	uint32_t okm = 0;
#pragma unroll
	for(int i = 0; i < 16; i++)
	{
		const int n = nfirst + 32 * i;
		bool ok;
		if(narrow)
			ok = (c.fmask >> kf) & 1u;
		else
		{
			const int64_t fr = (int64_t)c.fa + kf;
			ok = active && fr < a.valid_stride && vrow[fr] != 0;
		}
		ok = ok && n < c.stuck;
		const uint32_t bit0 = tin * U.bpt + U.boff0;
		const void *src = ok ? (const void *)((const uint32_t *)fp + (bit0 >> 5)) : (const void *)U.buf;
		cp_async4(stage_addr + (uint32_t)(i * kThreadsF + tid) * 4u, src, ok ? 4u : 0u);
		okm |= (uint32_t)ok << i;
		if(i < 15)
		{
			tin += 32u;
			while(tin >= U.fs)
			{
				tin -= U.fs;
				kf++;
				fp += U.framebytes;
			}
		}
	}
	asm volatile("cp.async.commit_group;\n" ::: "memory");
	return okm;
}

}  // namespace

__global__ void __launch_bounds__(kThreadsF, 2) k_fstage_tc(const FsArgs a, const uint4 *__restrict__ tables,
                                                         int count, int nunits, int32_t *err)
{
	extern __shared__ __align__(1024) unsigned char fsm_tc[];
	__shared__ float lut8[256];
	__shared__ float2 lut4[16];
	__shared__ TcFftConst fc[2][2];                 // [unit parity][time of the unit]
	__shared__ uint32_t okms[kThreadsF];            // valid-sample bits of each thread's staged words
	__shared__ TcUnit tus[2];                       // [unit parity] fields of the unit
	__shared__ uint64_t mb1, mb2, mbd;
	__shared__ uint32_t tmem_s;
	unsigned char *base = (unsigned char *)(((uintptr_t)fsm_tc + 1023) & ~(uintptr_t)1023);
	unsigned char *sB = base + kOffB;
	const float2 *stw = (const float2 *)(base + kOffTw);
	const uint32_t *stage = (const uint32_t *)(base + kOffStage);
	const uint32_t stage_addr = su32(base + kOffStage);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int order = a.order;
	constexpr int nchan = kN / 2;

	for(int i = tid; i < kTablesBytes / 16; i += kThreadsF)
		((uint4 *)base)[i] = __ldg(tables + i);
	for(int i = tid; i < 256; i += kThreadsF)
		lut8[i] = (float)((i - 128) / 3.3);               // format_vdif.c:122
	if(tid < 16)
		lut4[tid] = make_float2(level2f(tid & 3u), level2f(tid >> 2));
	if(tid == 0)
	{
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(su32(&mb1)));
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(su32(&mb2)));
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(su32(&mbd)));
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	if(warp == 0)
	{
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(su32(&tmem_s)),
		             "r"(256u));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
	}
	asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");      // tables -> tensor-core reads
	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	const uint32_t tmem = tmem_s;

	// prologue: constants and word loads of the first unit
	const int u0 = blockIdx.x;
	if(u0 < nunits)
	{
		if(tid == 0)
			tus[0] = tc_unit(a, u0, count);
		__syncthreads();
		const TcUnit &U = tus[0];
		if(warp < 2 && lane == 0)
		{
			const int t = U.t0 + warp;
			FftParam p;
			p.status = kFftZero;
			if(t < a.T)
				p = a.params[(int64_t)U.station * a.T + t];
			fc[0][warp] = tc_consts(U, p, t, a.T, order, a.fraclo);
		}
		__syncthreads();
		okms[tid] = tc_prefetch(a, U, fc[0][warp >> 2], stage_addr, warp, lane, tid);
	}

	int ku = 0;
	for(int u = u0; u < nunits; u += gridDim.x, ku++)
	{
		const int slot = ku & 1;
		const TcUnit &U = tus[slot];
		const int un = u + gridDim.x;
		const bool has_next = un < nunits;
		// the next unit's fields and FFT parameters (lanes 0 of warps 0, 1):
		// loads in flight during this decode
		TcUnit Un;
		FftParam pn;
		pn.status = kFftZero;
		if(has_next && warp < 2 && lane == 0)
		{
			Un = tc_unit(a, un, count);
			if(Un.t0 + warp < a.T)
				pn = a.params[(int64_t)Un.station * a.T + Un.t0 + warp];
		}
		asm volatile("cp.async.wait_all;\n" ::: "memory");
		__syncthreads();

		// ---- (b) decode x[32 n1 + n2] (n1 in this warp's quarter) from the
		// staged words into the operand of MMA 1: column (FFT = 2 time + band,
		// n2), K = (re|im, n1)
		{
			const int tl = warp >> 2, q4 = warp & 3, n2 = lane;
			const TcFftConst &c = fc[slot][tl];
			const uint32_t okm = okms[tid];
			const int nfirst = n2 + 32 * 16 * q4;
			const uint32_t xs = c.so + (uint32_t)nfirst;
			uint32_t kf = xs / U.fs, tin = xs - kf * U.fs;
			const uint8_t *fp = U.buf + ((int64_t)c.fa + kf) * U.framebytes + U.header;
			float ph = c.P0 + (float)nfirst * c.alpha;
			ph -= rintf(ph);
			float rr, ri;
			__sincosf(-6.283185307179586f * ph, &ri, &rr);
#pragma unroll
			for(int h = 0; h < 2; h++)
			{
				uint32_t re0[4], im0[4], re1[4], im1[4];
#pragma unroll
				for(int i2 = 0; i2 < 4; i2++)
				{
					float x0r[2], x0i[2], x1r[2], x1i[2];
#pragma unroll
					for(int e = 0; e < 2; e++)
					{
						const int i = 8 * h + 2 * i2 + e;
						float v0 = 0.0f, v1 = 0.0f;
						if((okm >> i) & 1u)
						{
							const uint32_t bit0 = tin * U.bpt + U.boff0;
							const uint32_t raw = stage[i * kThreadsF + tid];
							const uint32_t w0 = raw >> (bit0 & 31u);
							if(U.pair4)
							{
								const float2 l = lut4[w0 & 15u];
								v0 = l.x;
								v1 = l.y;
							}
							else
							{
								const uint32_t bit1 = tin * U.bpt + U.boff1;
								const uint32_t w1 = (U.oneword ? raw : __ldg((const uint32_t *)fp + (bit1 >> 5))) >> (bit1 & 31u);
								v0 = U.nbits == 2 ? level2f(w0 & 3u) : lut8[w0 & 255u];
								v1 = U.nbits == 2 ? level2f(w1 & 3u) : lut8[w1 & 255u];
							}
						}
						x0r[e] = v0 * rr;
						x0i[e] = v0 * ri;
						x1r[e] = v1 * rr;
						x1i[e] = v1 * ri;
						const float nr = rr * c.Ur - ri * c.Ui;
						ri = rr * c.Ui + ri * c.Ur;
						rr = nr;
						if(i < 15)
						{
							tin += 32u;
							while(tin >= U.fs)
							{
								tin -= U.fs;
								kf++;
								fp += U.framebytes;
							}
						}
					}
					re0[i2] = pack_h2(x0r[0], x0r[1]);
					im0[i2] = pack_h2(x0i[0], x0i[1]);
					re1[i2] = pack_h2(x1r[0], x1r[1]);
					im1[i2] = pack_h2(x1i[0], x1i[1]);
				}
				const int chunk = 2 * q4 + h;
				const int col0 = (tl * 2) * 32 + n2, col1 = col0 + 32;
				*(uint4 *)(sB + swz(col0, chunk)) = make_uint4(re0[0], re0[1], re0[2], re0[3]);
				*(uint4 *)(sB + 16384 + swz(col0, chunk)) = make_uint4(im0[0], im0[1], im0[2], im0[3]);
				*(uint4 *)(sB + swz(col1, chunk)) = make_uint4(re1[0], re1[1], re1[2], re1[3]);
				*(uint4 *)(sB + 16384 + swz(col1, chunk)) = make_uint4(im1[0], im1[1], im1[2], im1[3]);
			}
		}
		if(has_next && warp < 2 && lane == 0)
		{
			fc[slot ^ 1][warp] = tc_consts(Un, pn, Un.t0 + warp, a.T, order, a.fraclo);
			if(warp == 0)
				tus[slot ^ 1] = Un;
		}
		asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
		__syncthreads();
		// the next unit's word loads: in flight during the MMAs, twiddle and output
		if(has_next)
			okms[tid] = tc_prefetch(a, tus[slot ^ 1], fc[slot ^ 1][warp >> 2], stage_addr, warp, lane, tid);

		// ---- (c) MMA 1: D1[(k1, re|im)][(FFT, n2)], FP16 x FP16 -> FP32, M = N = 128
		if(tid == 0)
		{
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			const uint32_t idesc = (1u << 4) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
			const uint32_t aA = su32(base), aB = su32(sB);
#pragma unroll
			for(int kk = 0; kk < 8; kk++)
			{
				const uint32_t off = (uint32_t)((kk >> 2) * 16384 + (kk & 3) * 32);
				mma_f16(tmem, sdesc128(aA + off), sdesc128(aB + off), idesc, kk > 0 ? 1u : 0u);
			}
			commit_to(&mb1);
		}
		if(!__syncthreads_and(mbar_wait_f(&mb1, ku & 1)))
		{
			if(tid == 0)
				atomicExch(err, 7);
			break;
		}
		asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

		// ---- (d) twiddle w_N^(n2 k1) in FP32 (one rounding to FP16 per value);
		// rows (FFT, k1) of the MMA 2 operands
		{
			const int q = warp & 3, hcol = warp >> 2;
			const int r = 32 * q + lane, k1 = r >> 1, part = r & 1;
			const float sg = part ? 1.0f : -1.0f;                  // re lane subtracts o wi
#pragma unroll
			for(int cc = 0; cc < 2; cc++)
			{
				const int fftl = 2 * hcol + cc;
				float v[32];
				tld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * fftl), v);
				uint32_t pkv[16];
#pragma unroll
				for(int n2 = 0; n2 < 32; n2 += 2)
				{
					const float o0 = __shfl_xor_sync(0xffffffffu, v[n2], 1);
					const float o1 = __shfl_xor_sync(0xffffffffu, v[n2 + 1], 1);
					const float2 w0 = stw[n2 * kN1 + k1], w1 = stw[(n2 + 1) * kN1 + k1];
					pkv[n2 >> 1] = pack_h2(fmaf(sg * o0, w0.y, v[n2] * w0.x), fmaf(sg * o1, w1.y, v[n2 + 1] * w1.x));
				}
				const int R3 = fftl * 64 + k1;
				unsigned char *tile = sB + (R3 >> 7) * 16384;
				const int rr3 = R3 & 127;
#pragma unroll
				for(int cq = 0; cq < 4; cq++)
					*(uint4 *)(tile + swz(rr3, part * 4 + cq)) =
					    make_uint4(pkv[4 * cq], pkv[4 * cq + 1], pkv[4 * cq + 2], pkv[4 * cq + 3]);
			}
		}
		asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
		asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
		__syncthreads();

		// ---- (e) MMA 2: D3[(FFT, k1)][(re|im, k2)] for the sideband's 16 k2, M = 128, N = 32
		if(tid == 0)
		{
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			const uint32_t idesc = (1u << 4) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
			const uint32_t aB3 = su32(base + kOffB3 + (U.lsb ? kB3 : 0)), aA = su32(sB);
#pragma unroll
			for(int m = 0; m < 2; m++)
#pragma unroll
				for(int kk = 0; kk < 4; kk++)
					mma_f16(tmem + 128u + 32u * m, sdesc128(aA + m * 16384 + kk * 32), sdesc128(aB3 + kk * 32), idesc,
					        kk > 0 ? 1u : 0u);
			commit_to(&mb2);
		}
		if(!__syncthreads_and(mbar_wait_f(&mb2, ku & 1)))
		{
			if(tid == 0)
				atomicExch(err, 8);
			break;
		}
		asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

		// ---- (f) channels c = k1 + 64 j: fractional-sample rotation, half2 or
		// bf16x2 out, scaled by 2^-kTcSpecExp
		{
			const int q = warp & 3, m = warp >> 2;
			const int r = 32 * q + lane;
			const int fftl = 2 * m + (r >> 6), k1 = r & 63;
			const int tl = fftl >> 1, b = fftl & 1;
			float v[32];
			tld32(tmem + ((uint32_t)(32 * q) << 16) + 128u + 32u * m, v);
			const TcFftConst &c = fc[slot][tl];
			const int rw = b ? U.row1 : U.row0;
			if(c.t < a.T && rw >= 0)
			{
				const DevFreqPlan &P = a.plans[U.freq];
				const int64_t spec_off = P.spec_off;
				const int prow = P.nrow;
				const uint32_t tcb = (uint32_t)P.tcb, tnblk = (uint32_t)P.tnblk;
				float turns = (float)(U.lsb ? k1 - nchan : k1) * c.dfs + c.postf;
				turns -= rintf(turns);
				float qr, qi;
				__sincosf(6.283185307179586f * turns, &qi, &qr);
				constexpr float osc = 1.0f / (float)(1 << kTcSpecExp);
				qr *= osc;
				qi *= osc;
				// channel k1 + 64 j -> (block, position): start, then step by 64 channels
				const uint32_t PT = (uint32_t)prow * tcb;
				uint32_t blk = (uint32_t)k1 / tcb, cl = (uint32_t)k1 - blk * tcb;
				const uint32_t dblk = 64u / tcb, dcl = 64u - dblk * tcb;
				uint32_t off = blk * PT + cl;
				uint32_t *o = (uint32_t *)a.spec + spec_off + ((int64_t)c.t * tnblk * prow + rw) * tcb;
				const bool h16 = a.h16 != 0;
#pragma unroll
				for(int j = 0; j < 16; j++)
				{
					const float xr = v[j], xi = v[16 + j];
					const float yr = xr * qr - xi * qi, yi = xr * qi + xi * qr;
					if(h16)
						o[off] = pack_h2(yr, yi);
					else
					{
						const __nv_bfloat162 b = __floats2bfloat162_rn(yr, yi);
						o[off] = *(const uint32_t *)&b;
					}
					const float nr = qr * c.Rr - qi * c.Ri;
					qi = qr * c.Ri + qi * c.Rr;
					qr = nr;
					cl += dcl;
					off += dblk * PT + dcl;
					if(cl >= tcb)
					{
						cl -= tcb;
						off += PT - tcb;
					}
				}
			}
		}
		asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
		__syncthreads();
	}
	// copies still in flight (error path) land before the CTA exits
	asm volatile("cp.async.wait_all;\n" ::: "memory");
	// every MMA issued by thread 0 has completed once mbd arrives
	if(tid == 0)
	{
		commit_to(&mbd);
		if(!mbar_wait_f(&mbd, 0))
			atomicExch(err, 9);
	}
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	if(warp == 0)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(256u));
}

// ---------------------------------------------------------------- host side
// Constant tables in the kernel's shared-memory byte layout (values in double,
// rounded once): DFT-64 rows (k1, re|im) over K = (re|im, n1); DFT-32
// columns (re|im, k2) over K = (re|im, n2) for k2 in [0, 16) (upper sideband)
// and [16, 32) (lower); twiddles w_2048^(n2 k1) as float2 [n2][k1].
size_t fstage_tc_tables_bytes() { return kTablesBytes; }

void make_fstage_tc_tables(void *out)
{
	unsigned char *o = (unsigned char *)out;
	memset(o, 0, kTablesBytes);
	auto put = [&](unsigned char *tile, int row, int kin, double v) {
		const int chunk = kin >> 3;
		const int off = row * 128 + ((chunk ^ (row & 7)) << 4) + (kin & 7) * 2;
		const __half h = __double2half(v);
		memcpy(tile + off, &h, 2);
	};
	for(int k1 = 0; k1 < kN1; k1++)
		for(int n1 = 0; n1 < kN1; n1++)
		{
			const double th = 2.0 * M_PI * (double)(k1 * n1 % kN1) / kN1;
			const double c = cos(th), sn = sin(th);
			put(o, 2 * k1, n1, c);                  // re out: [cos | sin]
			put(o + 16384, 2 * k1, n1, sn);
			put(o, 2 * k1 + 1, n1, -sn);            // im out: [-sin | cos]
			put(o + 16384, 2 * k1 + 1, n1, c);
		}
	for(int side = 0; side < 2; side++)
	{
		unsigned char *t = o + kOffB3 + side * kB3;
		for(int j = 0; j < 16; j++)
		{
			const int k2 = 16 * side + j;
			for(int n2 = 0; n2 < kN2; n2++)
			{
				const double ph = 2.0 * M_PI * (double)(n2 * k2 % kN2) / kN2;
				const double c = cos(ph), sn = sin(ph);
				put(t, j, n2, c);                   // re out: [cos | sin]
				put(t, j, 32 + n2, sn);
				put(t, 16 + j, n2, -sn);            // im out: [-sin | cos]
				put(t, 16 + j, 32 + n2, c);
			}
		}
	}
	// twiddles w_2048^(n2 k1) as float2 [n2][k1]
	float2 *tw = (float2 *)(o + kOffTw);
	for(int n2 = 0; n2 < kN2; n2++)
		for(int k1 = 0; k1 < kN1; k1++)
		{
			const double ang = -2.0 * M_PI * (double)(n2 * k1) / kN;
			tw[n2 * kN1 + k1] = make_float2((float)cos(ang), (float)sin(ang));
		}
}

bool fstage_tc_eligible(int N, int order, bool any_lsb)
{
	return N == kN && (order == 1 || (order == 0 && !any_lsb));
}

void launch_fstage_tc(const FKind &k, FsArgs a, int nsm, cudaStream_t stream)
{
	if(k.count <= 0 || a.T <= 0 || !k.tctab)
		return;
	a.first = k.first;
	const int nunits = k.count * ((a.T + 1) / 2);
	cudaFuncSetAttribute(k_fstage_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemTc);
	cudaFuncSetAttribute(k_fstage_tc, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
	int grid = 2 * nsm;
	if(grid > nunits)
		grid = nunits;
	k_fstage_tc<<<grid, kThreadsF, kSmemTc, stream>>>(a, (const uint4 *)k.tctab, k.count, nunits, a.err);
}

}  // namespace fxb
