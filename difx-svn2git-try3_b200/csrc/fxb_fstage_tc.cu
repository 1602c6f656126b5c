// F stage of the tensor-core form with the FFT on the tensor cores (sm_100a).
//
// Mode::process (mpifxcorr/src/mode.cpp:845-1308) per FFT of N = 2048 points:
// VDIF decode, fringe rotation, complex FFT, sideband selection and
// fractional-sample rotation.  The FFT runs as the four-step factorisation
// N = 32 x 64 (n = 64 n1 + n2, k = k1 + 32 k2):
//   Y[k1][n2] = sum_n1 x[64 n1 + n2] w_32^(n1 k1)        (MMA 1)
//   Z[k1][n2] = Y[k1][n2] w_2048^(n2 k1)                 (CUDA cores, FP32)
//   X[k1 + 32 k2] = sum_n2 Z[k1][n2] w_64^(n2 k2)         (MMA 2, the 32 k2 of the sideband)
// with complex products written as real ones.  Operands are FP16 (11-bit
// significands), accumulation FP32 in tensor memory; the samples, the
// twiddled intermediate and the output are each rounded to FP16 once.
//
// A work unit is one station at one FFT time with two subbands of equal
// sideband (four FFTs: subband sb, polarisation p, channel ch = 2 sb + p).
//   MMA 1: A = samples, MN-major (M = 128 rows (p, n2) per subband, K = 64 =
//          (re|im, n1)); B = the real-ified DFT-32 (N = 64 = (k1, re|im)),
//          K-major.  One thread (tensor-memory lane (p, n2)) then holds
//          Y[.][n2] of both parts for all k1.
//   MMA 2: A = Z, MN-major (M = 128 rows (ch, k1), K = 128 = (re|im, n2));
//          B = the real-ified DFT-64 columns of the sideband (N = 64 =
//          (k2, re|im)), K-major.  Lane (ch, k1) holds channels k1 + 32 k2.
// MN-major operands let each thread store 16-byte runs: the decode writes 8
// consecutive times n2 of one n1, the twiddle 8 consecutive k1 of one n2.
//
// Persistent CTAs (one per SM, 18 warps at 96 registers: an SM sub-partition
// holds at most five of them in its 16384 registers), warp-specialised:
//   warp 17     producer: builds the records of 32 units at a time (one lane
//               per unit: pair, FFT parameters, fringe and fractional-sample
//               constants, output offsets) into a shared-memory ring and
//               stages each unit's VDIF window into shared memory (bulk
//               copies of the valid frames),
//   warps 0-7   decode: 8 consecutive times -> the fringe-rotated FP16
//               samples of the unit's four channels (two-time lookup of
//               both polarisations, FP32 rotation),
//   warps 8-11  twiddle: D1 (tensor memory, 32 columns at a time) -> Z (FP16
//               operand, in the operand buffer MMA 1 has finished with),
//   warps 12-15 output: D2 (32 columns at a time) -> fractional-sample
//               rotation -> FP16 (or BF16) spectra,
//   warp 16     MMA issuer (one thread).
// Three operand buffers and two tensor-memory slots (D1 + D2 per slot)
// keep decode, MMAs, twiddle and output of different units overlapped.
// Every wait is bounded; a timeout sets the error flag, the CTA stops,
// waits (bounded) for its copies and MMAs in flight and frees its tensor
// memory.

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

constexpr int kN = 2048, kN1 = 32, kN2 = 64;
constexpr int kNS = 3;                          // operand buffers
constexpr int kOpBytes = 32768;                 // A1 (two 16 KB tiles) or A2 (32 KB)
constexpr int kB1Bytes = 64 * 128;              // DFT-32: 64 rows x 128 bytes (K = 64)
constexpr int kB2Bytes = 2 * 64 * 128;          // DFT-64 of one sideband: 2 K halves x 64 rows x 128 bytes
constexpr int kOffB1 = 0, kOffB2 = kB1Bytes;
constexpr int kTablesBytes = kOffB2 + 2 * kB2Bytes;
constexpr int kOffOp = kTablesBytes;            // 1024-aligned
// warp roles: kDecW decode warps, then 4 twiddle and 4 output warps (each
// set covers the four tensor-memory lane quadrants, warp % 4), the MMA warp
// and the producer warp
constexpr int kDecW = 8;
constexpr int kTwW0 = kDecW, kOutW0 = kDecW + 4, kMmaW = kDecW + 8, kProdW = kDecW + 9;
constexpr int kThreadsTc = 32 * (kDecW + 10);
static_assert(kTwW0 % 4 == 0 && kOutW0 % 4 == 0 && 8 % kDecW == 0, "warp roles");
constexpr uint32_t kWaitLimitF = 1u << 22;
constexpr int kTmemCols = 512;

static_assert(kOffOp % 1024 == 0, "operand buffers must be 1024-aligned");

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(su32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(su32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(su32(bar)), "r"(bytes) : "memory");
}

// bounded wait for the phase with parity `parity`; gives up early once
// another role has recorded a failure
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *fail)
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
		if((it & 255u) == 255u && *fail)
			return false;
	}
	return false;
}

// global -> shared bulk copy (both addresses and the size multiples of 16),
// completion counted in bytes on the mbarrier
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
	asm volatile(
	    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(su32(dst)),
	    "l"(src), "r"(bytes), "r"(su32(bar))
	    : "memory");
}

// shared-memory matrix descriptors (tcgen05 version 1, 128-byte swizzle)
// K-major: rows of 128 bytes, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t desc_k128(uint32_t saddr)
{
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3FFF);
	d |= (uint64_t)1 << 16;
	d |= (uint64_t)(1024 >> 4) << 32;
	d |= (uint64_t)1 << 46;
	d |= (uint64_t)2 << 61;
	return d;
}
// MN-major: 1024-byte atoms of 8 K rows x 64 MN values; the two MN atoms of
// a 128-row tile 1024 bytes apart (leading byte offset), K atoms 2048 bytes
// apart (stride byte offset)
__device__ __forceinline__ uint64_t desc_mn128(uint32_t saddr)
{
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3FFF);
	d |= (uint64_t)(1024 >> 4) << 16;
	d |= (uint64_t)(2048 >> 4) << 32;
	d |= (uint64_t)1 << 46;
	d |= (uint64_t)2 << 61;
	return d;
}

// byte offset of element (m, k) in a 128-row MN-major tile laid out
// [k / 8][m / 64][k % 8][128 bytes] with the 128-byte swizzle
__device__ __forceinline__ uint32_t mn_off(int m, int k)
{
	const int r = k & 7;
	return (uint32_t)((k >> 3) * 2048 + (m >> 6) * 1024 + r * 128 + ((((m & 63) >> 3) ^ r) << 4) + (m & 7) * 2);
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
#pragma unroll
	for(int i = 0; i < 32; i++)
		v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_h2(float a, float b)
{
	const __half2 h = __floats2half2_rn(a, b);
	return *(const uint32_t *)&h;
}

// one spectral value of the tensor-core forms: (re, im) as half2 or bf16x2
__device__ __forceinline__ uint32_t pack_spec(bool h16, float re, float im)
{
	if(h16)
		return pack_h2(re, im);
	const __nv_bfloat162 b = __floats2bfloat162_rn(re, im);
	return *(const uint32_t *)&b;
}

__device__ __forceinline__ float level2f(uint32_t code)
{
	const float mag = ((code ^ (code >> 1)) & 1u) ? 1.0f : 3.3359f;
	return (code & 2u) ? mag : -mag;
}

__device__ __forceinline__ float fracc(double x) { return (float)(x - rint(x)); }

// Everything the roles need of one work unit, built by the producer warp
// (one lane per unit, 32 units at a time) into a shared-memory ring.
struct UnitRec {
	float P0[2], alpha[2];        // fringe phase (turns) at n = 0 and per sample, per subband
	float Sr[2], Si[2];           // rotator step per sample exp(-2 pi i alpha)
	uint32_t fmask;               // validity of the window's frames (bit j: frame fa + j)
	int32_t so, fs;               // window start within frame fa, samples per frame
	int32_t swbits;               // staged bit of sample 0
	int32_t nib[2];               // 4-bit field of each subband's two bands in a time
	int32_t flags;                // kOk, kAllValid, kManual, kHas0, kHas1, kLsb0, kLsb1
	uint32_t fa;                  // first frame of the window
	int64_t a0;                   // first staged byte of the payloads from frame fa on
	int32_t nstage, station;      // staged bytes; station
	int32_t t;                    // FFT time
	float dhi[2][2], dlo[2][2];   // fractional-sample turns per channel of [subband][polarisation] (split_turns)
	float st32[2][2];             // the same over 32 channels, reduced to [-1/2, 1/2)
	float post[2][2];             // order-0 post-F turns plus the phase-offset rotation, per [subband][polarisation]
	int32_t row[2][2];            // spectra row of [subband][polarisation] (-1: not written)
	int64_t spec[2];              // first spectra value of the subband's [t][block][row][tcb] block
	int32_t tnblk[2], nrow[2], tcb[2];
};
enum : int32_t { kOk = 1, kAllValid = 2, kManual = 4, kHas0 = 8, kHas1 = 16, kLsb0 = 32, kLsb1 = 64 };
constexpr int kRing = 16;         // unit records in flight (>= staging + operand buffers + 2, with margin)
constexpr int kNStg = 3;          // VDIF staging buffers

template <int BPT>
struct TcLayout {
	static constexpr int kStgBytes = kN * BPT / 8 + 64;   // one window, 16-byte slack either side
	static constexpr int kOffStg = kOffOp + kNS * kOpBytes;
	static constexpr int kOffLut = kOffStg + kNStg * kStgBytes;
	static constexpr int kOffTw = kOffLut + 256 * 16;     // twiddles w_2048^(n2 k1), float2 [k1][n2]
	static constexpr int kOffRing = kOffTw + kN1 * kN2 * 8;
	// per output warp and lane: the spectra offset of channel k1 + 32 j (j = 0..31)
	// in the blocked layout of the last (tcb, nrow) seen
	static constexpr int kOffOutTab = (kOffRing + kRing * (int)sizeof(UnitRec) + 15) & ~15;
	static constexpr int kUsed = kOffOutTab + 4 * 32 * 32 * 4;
	static constexpr size_t kSmem = 1024 + (size_t)kUsed;
	static_assert(kOffStg % 16 == 0 && kStgBytes % 16 == 0, "staging must be 16-aligned");
	static_assert(kSmem <= 227 * 1024, "shared memory");
};

// the producer lane's record of unit k (u = blockIdx.x + k gridDim.x)
template <int BPT>
__device__ __forceinline__ UnitRec build_unit(const FsArgs &a, const int32_t *pairs, int npairs, int u)
{
	constexpr int nchan = kN / 2;
	UnitRec r;
	memset(&r, 0, sizeof(r));
	r.Sr[0] = r.Sr[1] = 1.0f;
	const int pi = u % npairs;
	r.t = u / npairs;
	const int gi[2] = {pairs[2 * pi], pairs[2 * pi + 1]};
	const FGroup g0 = a.groups[gi[0]];
	const int s = g0.station;
	r.station = s;
	const DevStation *Sp = a.st + s;
	const FftParam p = a.params[(int64_t)s * a.T + r.t];
	r.fs = Sp->framesamples;
	const double bw = Sp->bw;
	for(int sb = 0; sb < 2; sb++)
	{
		r.row[sb][0] = r.row[sb][1] = -1;
		if(gi[sb] < 0)
			continue;
		const FGroup g = sb == 0 ? g0 : a.groups[gi[sb]];
		const DevFreqPlan &P = a.plans[g.freq];
		r.flags |= (sb == 0 ? kHas0 : kHas1) | (g.lsb ? (sb == 0 ? kLsb0 : kLsb1) : 0);
		r.nib[sb] = g.band[0] >> 1;
		r.row[sb][0] = g.row[0];
		r.row[sb][1] = g.row[1];
		r.spec[sb] = P.spec_off + (int64_t)r.t * P.tnblk * P.nrow * P.tcb;
		r.tnblk[sb] = P.tnblk;
		r.nrow[sb] = P.nrow;
		r.tcb[sb] = P.tcb;
		if(p.status != kFftOk)
			continue;
		const double lo = g.lofreq;
		const int idl = p.integerdelay;
		// LO offset (mode.cpp:873-882, 932-951, 1061-1070): seconds since the
		// job start of the FFT's first sample (the scan starts with the job)
		const double walls = (double)a.sub[s].subsec + a.sub[s].subns / 1.0e9 +
		                     (double)r.t * kN * Sp->sampletime / 1.0e6;
		double postf = 0.0;
		if(a.order == 1)
		{
			const double fl = a.fraclo ? (lo - (int)lo) * (double)idl : 0.0;
			const double low = g.corr ? looff_wall_turns(g.looff, walls) : 0.0;
			r.P0[sb] = fracc(lo * p.b + fl + low);
			r.alpha[sb] = (float)(lo * p.a * (1.0 / kN) - g.looff * Sp->sampletime / 1.0e6);
			float sn, cs;
			sincospif(-2.0f * r.alpha[sb], &sn, &cs);
			r.Sr[sb] = cs;
			r.Si[sb] = sn;
		}
		else if(a.order == 0)
		{
			double pr0 = (p.averagedelay - idl) * lo;
			if(a.fraclo)
				pr0 += idl * (lo - (int)lo);
			pr0 -= walls * g.looff;
			postf = -(double)(float)(pr0 - (int)pr0);
		}
		// per polarisation: fse - clock offset (mode.cpp:1053-1059, 1099-1106)
		// and the phase-offset rotation (mode.cpp:1336-1347)
		for(int q = 0; q < 2; q++)
		{
			const double D = bw * (1.0 / nchan) * ((double)p.fse - g.clk[q]);
			split_turns(D, r.dhi[sb][q], r.dlo[sb][q]);
			r.st32[sb][q] = fracc(32.0 * D);
			r.post[sb][q] = (float)(postf + (double)g.phase[q]);
		}
	}
	if(p.status == kFftOk)
	{
		r.flags |= kOk;
		const uint32_t g = (uint32_t)p.nearest;
		r.fa = g / (uint32_t)r.fs;
		r.so = (int32_t)(g - r.fa * (uint32_t)r.fs);
		r.fmask = p.fmask;
		const int nwf = (r.so + kN - 1) / r.fs + 1;
		if(nwf < 32 ? (r.fmask == (1u << nwf) - 1u) : r.fmask == 0xFFFFFFFFu)
			r.flags |= kAllValid;
		// the window's times [so, so + N) of the payloads from frame fa on, 16-byte aligned
		const int64_t b0 = (int64_t)r.so * BPT, b1 = (int64_t)(r.so + kN) * BPT;
		r.a0 = (b0 >> 3) & ~(int64_t)15;
		const int64_t a1 = (((b1 + 7) >> 3) + 15) & ~(int64_t)15;
		r.swbits = (int32_t)(b0 - 8 * r.a0);
		r.nstage = (int32_t)(a1 - r.a0);
		if(((uintptr_t)a.sub[s].buf & 15u) != 0)
			r.flags |= kManual;
	}
	return r;
}

}  // namespace

// tables: DFT-32 (B of MMA 1), DFT-64 upper and lower sideband (B of MMA 2),
// in their shared-memory byte layouts.  pairs: [npairs][2] FGroup indices of
// the two subbands of a work unit (-1: none); unit u = pair u % npairs at
// FFT time u / npairs.  BPT: bits per time of the stations' VDIF words
// (2-bit bands: 2 x bands).
template <int BPT, bool H16>
__global__ void __launch_bounds__(kThreadsTc, 1) k_fstage_tc(const FsArgs a, const uint4 *__restrict__ tables,
                                                          const int32_t *__restrict__ pairs, int npairs, int nunits,
                                                          int32_t *err)
{
	using LY = TcLayout<BPT>;
	extern __shared__ __align__(1024) unsigned char fsm_tc[];
	__shared__ uint64_t stg_full[kNStg], stg_empty[kNStg], op_full[kNS], op_empty[kNS], d1_full[2], d1_empty[2],
	    a2_full[2], d2_full[2], d2_empty[2], mma_done;
	__shared__ uint32_t tmem_s;
	__shared__ volatile int fail_s;
	__shared__ int stg_issued_s, stg_used_s;
	unsigned char *base = (unsigned char *)(((uintptr_t)fsm_tc + 1023) & ~(uintptr_t)1023);
	unsigned char *ops = base + kOffOp;
	unsigned char *stg = base + LY::kOffStg;
	float4 *lut = (float4 *)(base + LY::kOffLut);
	float2 *twt = (float2 *)(base + LY::kOffTw);
	UnitRec *ring = (UnitRec *)(base + LY::kOffRing);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int order = a.order;
	constexpr int nchan = kN / 2;
	const int nk = ((int)blockIdx.x < nunits) ? (nunits - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;

	for(int i = tid; i < kTablesBytes / 16; i += blockDim.x)
		((uint4 *)base)[i] = __ldg(tables + i);
	// two times of both polarisations of one subband: index = nibble(t) |
	// nibble(t + 1) << 4, nibble = code(p0) | code(p1) << 2 (format_vdif.c:78)
	for(int i = tid; i < 256; i += blockDim.x)
		lut[i] = make_float4(level2f(i & 3u), level2f((i >> 4) & 3u), level2f((i >> 2) & 3u), level2f((i >> 6) & 3u));
	for(int i = tid; i < kN1 * kN2; i += blockDim.x)
	{
		const int k1 = i / kN2, n2 = i - k1 * kN2;
		float sn, cs;
		sincospif(-(float)(n2 * k1) / (float)(kN / 2), &sn, &cs);
		twt[i] = make_float2(cs, sn);
	}
	if(tid == 0)
	{
		for(int i = 0; i < kNStg; i++)
		{
			mbar_init(&stg_full[i], 1);
			mbar_init(&stg_empty[i], kDecW);
		}
		for(int i = 0; i < 2; i++)
		{
			mbar_init(&d1_full[i], 1);
			mbar_init(&d1_empty[i], 4);
			mbar_init(&a2_full[i], 4);
			mbar_init(&d2_full[i], 1);
			mbar_init(&d2_empty[i], 4);
		}
		for(int i = 0; i < kNS; i++)
		{
			mbar_init(&op_full[i], kDecW);
			mbar_init(&op_empty[i], 1);
		}
		mbar_init(&mma_done, 1);
		fail_s = 0;
		stg_issued_s = 0;
		stg_used_s = 0;
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	if(warp == kMmaW)
	{
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(su32(&tmem_s)),
		             "r"((uint32_t)kTmemCols));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
	}
	asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");      // tables -> tensor-core reads
	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	const uint32_t tmem = tmem_s;

	if(warp == kProdW)
	{
		// ================================================================ producer
		bool ok = true;
		for(int kb = 0; kb < nk && ok; kb += 32)
		{
			UnitRec r;
			if(kb + lane < nk)
				r = build_unit<BPT>(a, pairs, npairs, (int)blockIdx.x + (kb + lane) * (int)gridDim.x);
			for(int i = 0; i < 32 && kb + i < nk; i++)
			{
				const int k = kb + i, slot = k % kNStg;
				// every lane takes the same decision (the warp meets at __syncwarp below)
				const bool okw = k < kNStg || mbar_wait(&stg_empty[slot], (uint32_t)((k / kNStg) - 1) & 1u, &fail_s);
				if(!__all_sync(0xffffffffu, okw))
				{
					fail_s = 10;
					ok = false;
					break;
				}
				if(lane == i)
				{
					ring[k % kRing] = r;
					uint32_t want = 0;
					const bool copy = (r.flags & kOk) && !(r.flags & kManual);
					const int nwf = (r.so + kN - 1) / r.fs + 1;
					const DevStation *Sp = a.st + r.station;
					const int P = Sp->payload;
					const int64_t a1 = r.a0 + r.nstage;
					for(int j = 0; copy && j < nwf && j < 32; j++)
					{
						const int64_t f0 = (int64_t)j * P, lo_ = r.a0 > f0 ? r.a0 : f0, hi_ = a1 < f0 + P ? a1 : f0 + P;
						if(hi_ > lo_ && ((r.fmask >> j) & 1u))
							want += (uint32_t)(hi_ - lo_);
					}
					if(want)
					{
						// the byte count is armed before the copies that complete it
						mbar_expect_tx(&stg_full[slot], want);
						unsigned char *dst = stg + slot * LY::kStgBytes;
						const uint8_t *buf = a.sub[r.station].buf;
						for(int j = 0; j < nwf && j < 32; j++)
						{
							const int64_t f0 = (int64_t)j * P, lo_ = r.a0 > f0 ? r.a0 : f0, hi_ = a1 < f0 + P ? a1 : f0 + P;
							if(hi_ <= lo_ || !((r.fmask >> j) & 1u))
								continue;
							const uint8_t *src = buf + ((int64_t)r.fa + j) * Sp->framebytes + Sp->header + (lo_ - f0);
							bulk_g2s(dst + (lo_ - r.a0), src, (uint32_t)(hi_ - lo_), &stg_full[slot]);
						}
					}
					else
						mbar_arrive(&stg_full[slot]);
					stg_issued_s = k + 1;
				}
				__syncwarp();
			}
		}
	}
	else if(warp < kDecW)
	{
		// ================================================================ decode
		const int dt = tid;
		for(int k = 0; k < nk; k++)
		{
			const int slot = k % kNStg, s = k % kNS;
			bool okw = mbar_wait(&stg_full[slot], (uint32_t)(k / kNStg) & 1u, &fail_s);
			if(okw && k >= kNS)
				okw = mbar_wait(&op_empty[s], (uint32_t)((k / kNS) - 1) & 1u, &fail_s);
			if(!__all_sync(0xffffffffu, okw))      // the warp leaves together
			{
				fail_s = 11;
				break;
			}
			if(dt == 0)
				stg_used_s = k + 1;
			const UnitRec &R = ring[k % kRing];
			const int flags = R.flags;
			unsigned char *A1 = ops + s * kOpBytes;
			const uint32_t *words = (const uint32_t *)(stg + slot * LY::kStgBytes);
			if((flags & kOk) && (flags & kManual))
			{
				// station buffer without 16-byte alignment: every decode warp copies the
				// window's valid frames with byte loads (the same values, so the warps
				// may overlap) before reading it
				const DevStation *Sp = a.st + R.station;
				const uint8_t *buf = a.sub[R.station].buf;
				uint32_t *sw_ = (uint32_t *)(stg + slot * LY::kStgBytes);
				for(int i = lane; i < R.nstage / 4; i += 32)
				{
					const int64_t c = R.a0 + 4 * (int64_t)i;
					const int j = (int)(c / Sp->payload);
					uint32_t v = 0u;
					if(j < 32 && ((R.fmask >> j) & 1u))
					{
						const uint8_t *b = buf + ((int64_t)R.fa + j) * Sp->framebytes + Sp->header + (c - (int64_t)j * Sp->payload);
						v = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
					}
					sw_[i] = v;
				}
				__syncwarp();
			}
			const int so = R.so, fs = R.fs, swbits = R.swbits;
			const uint32_t fmask = R.fmask;
#pragma unroll 1
			for(int it = 0; it < 8 / kDecW; it++)
			{
				const int item = dt + 32 * kDecW * it;
				const int n1 = item >> 3, g = item & 7;
				const int n0 = 64 * n1 + 8 * g;             // first time of the item
				// the item's 8 times (bits swbits + n0 BPT ..) as NW aligned 32-bit
				// words, from the covering 16-byte quads of the staged window
				constexpr int NW = BPT / 4 > 1 ? BPT / 4 : 1;      // words of 8 times
				constexpr int NQ = (3 + NW + 1 + 3) / 4;            // quads that cover them from any start
				const int bitpos = swbits + n0 * BPT;
				const int wq = (bitpos >> 5) & ~3;
				const int ws = (bitpos >> 5) - wq, bs = bitpos & 31;
				uint32_t all[4 * NQ];
#pragma unroll
				for(int q = 0; q < NQ; q++)
				{
					const uint4 v4 = *(const uint4 *)(words + wq + 4 * q);
					all[4 * q] = v4.x;
					all[4 * q + 1] = v4.y;
					all[4 * q + 2] = v4.z;
					all[4 * q + 3] = v4.w;
				}
				uint32_t w[NW];
				switch(ws)
				{
				case 0:
#pragma unroll
					for(int i = 0; i < NW; i++) w[i] = __funnelshift_r(all[i], all[i + 1], bs);
					break;
				case 1:
#pragma unroll
					for(int i = 0; i < NW; i++) w[i] = __funnelshift_r(all[i + 1], all[i + 2], bs);
					break;
				case 2:
#pragma unroll
					for(int i = 0; i < NW; i++) w[i] = __funnelshift_r(all[i + 2], all[i + 3], bs);
					break;
				default:
#pragma unroll
					for(int i = 0; i < NW; i++) w[i] = __funnelshift_r(all[i + 3], all[i + 4], bs);
					break;
				}
				// per-time validity (frames of the window that were not copied read as zero)
				uint32_t vm = (flags & kOk) ? 0xFFu : 0u;
				if((flags & kOk) && !(flags & kAllValid))
				{
					vm = 0u;
					const int x0 = so + n0;
					int kf = x0 / fs;
					int nb = (kf + 1) * fs - so;                // first time of the next frame
#pragma unroll
					for(int j = 0; j < 8; j++)
					{
						if(n0 + j >= nb)
						{
							kf++;
							nb += fs;
						}
						vm |= (kf < 32 ? ((fmask >> kf) & 1u) : 0u) << j;
					}
				}
#pragma unroll 1
				for(int sb = 0; sb < 2; sb++)
				{
					const int nsh = 4 * R.nib[sb];
					const uint32_t vms = (flags & (sb == 0 ? kHas0 : kHas1)) ? vm : 0u;
					float dv0[8], dv1[8];
#pragma unroll
					for(int j = 0; j < 8; j += 2)
					{
						// nibble of time j: bits j BPT + nsh of the item's words (for 64
						// bits per time the subband's word of the time pair is picked by nsh)
						uint32_t wa, wb;
						int sa, sb2;
						if constexpr(BPT <= 32)
						{
							wa = w[(j * BPT) >> 5];
							wb = w[((j + 1) * BPT) >> 5];
							sa = ((j * BPT) & 31) + nsh;
							sb2 = (((j + 1) * BPT) & 31) + nsh;
						}
						else
						{
							const bool hi = nsh >= 32;
							wa = hi ? w[2 * j + 1] : w[2 * j];
							wb = hi ? w[2 * j + 3] : w[2 * j + 2];
							sa = sb2 = nsh & 31;
						}
						const uint32_t idx = ((wa >> sa) & 15u) | (((wb >> sb2) & 15u) << 4);
						const float4 l = lut[idx];
						const bool v0 = (vms >> j) & 1u, v1 = (vms >> (j + 1)) & 1u;
						dv0[j] = v0 ? l.x : 0.0f;
						dv0[j + 1] = v1 ? l.y : 0.0f;
						dv1[j] = v0 ? l.z : 0.0f;
						dv1[j + 1] = v1 ? l.w : 0.0f;
					}
					// fringe rotator exp(-2 pi i (P0 + alpha n)) at n = n0 .. n0 + 7
					const float Sr = R.Sr[sb], Si = R.Si[sb];
					float rr = 1.0f, ri = 0.0f;
					if(order == 1)
					{
						float ph = R.P0[sb] + R.alpha[sb] * (float)n0;
						ph -= rintf(ph);
						__sincosf(-6.283185307179586f * ph, &ri, &rr);
					}
					uint32_t re0[4], im0[4], re1[4], im1[4];
#pragma unroll
					for(int j = 0; j < 8; j += 2)
					{
						const float rr1 = rr * Sr - ri * Si;
						const float ri1 = rr * Si + ri * Sr;
						re0[j >> 1] = pack_h2(dv0[j] * rr, dv0[j + 1] * rr1);
						im0[j >> 1] = pack_h2(dv0[j] * ri, dv0[j + 1] * ri1);
						re1[j >> 1] = pack_h2(dv1[j] * rr, dv1[j + 1] * rr1);
						im1[j >> 1] = pack_h2(dv1[j] * ri, dv1[j + 1] * ri1);
						rr = rr1 * Sr - ri1 * Si;
						ri = rr1 * Si + ri1 * Sr;
					}
					// A1 tile sb: rows m = p 64 + n2 (the 8 times 8g..8g+7 are one 16-byte
					// run), K = part 32 + n1
					unsigned char *T1 = A1 + sb * 16384;
					const uint32_t ore = mn_off(8 * g, n1), oim = mn_off(8 * g, 32 + n1);
					*(uint4 *)(T1 + ore) = make_uint4(re0[0], re0[1], re0[2], re0[3]);
					*(uint4 *)(T1 + oim) = make_uint4(im0[0], im0[1], im0[2], im0[3]);
					*(uint4 *)(T1 + ore + 1024) = make_uint4(re1[0], re1[1], re1[2], re1[3]);
					*(uint4 *)(T1 + oim + 1024) = make_uint4(im1[0], im1[1], im1[2], im1[3]);
				}
			}
			asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
			__syncwarp();
			if(lane == 0)
			{
				mbar_arrive(&op_full[s]);
				mbar_arrive(&stg_empty[slot]);
			}
		}
	}
	else if(warp < kOutW0)
	{
		// ================================================================ twiddle
		const int L = tid - 32 * kTwW0;         // tensor-memory lane (p, n2)
		const int p = L >> 6, n2 = L & 63;
		const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
		const float2 *tw = twt + n2;             // w_2048^(n2 k1) at tw[k1 kN2]
		for(int k = 0; k < nk; k++)
		{
			const int b = k & 1, s = k % kNS;
			if(!__all_sync(0xffffffffu, mbar_wait(&d1_full[b], (uint32_t)(k >> 1) & 1u, &fail_s)))
			{
				fail_s = 12;
				break;
			}
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			unsigned char *A2 = ops + s * kOpBytes;
#pragma unroll 1
			for(int h = 0; h < 4; h++)
			{
				// subband sb, channels k1 in [16 hh, 16 hh + 16): 32 columns
				const int sb = h >> 1, hh = h & 1;
				float v[32];
				tld32(tmem + lane_base + (uint32_t)(256 * b + 64 * sb + 32 * hh), v);
				tld_wait();
				// Z[k1][n2] = Y[k1][n2] w^(n2 k1); A2 row m = ch 32 + k1 with ch = 2 sb + p,
				// K = part 64 + n2
				const int m0 = (2 * sb + p) * 32 + 16 * hh;
				uint32_t zr[8], zi[8];
#pragma unroll
				for(int q = 0; q < 16; q += 2)
				{
					const int k1 = 16 * hh + q;
					const float y0r = v[2 * q], y0i = v[2 * q + 1], y1r = v[2 * q + 2], y1i = v[2 * q + 3];
					const float2 w0 = tw[k1 * kN2], w1 = tw[(k1 + 1) * kN2];
					zr[q >> 1] = pack_h2(y0r * w0.x - y0i * w0.y, y1r * w1.x - y1i * w1.y);
					zi[q >> 1] = pack_h2(y0r * w0.y + y0i * w0.x, y1r * w1.y + y1i * w1.x);
				}
#pragma unroll
				for(int c = 0; c < 2; c++)
				{
					*(uint4 *)(A2 + mn_off(m0 + 8 * c, n2)) = make_uint4(zr[4 * c], zr[4 * c + 1], zr[4 * c + 2], zr[4 * c + 3]);
					*(uint4 *)(A2 + mn_off(m0 + 8 * c, 64 + n2)) =
					    make_uint4(zi[4 * c], zi[4 * c + 1], zi[4 * c + 2], zi[4 * c + 3]);
				}
			}
			asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
			asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
			__syncwarp();
			if(lane == 0)
			{
				mbar_arrive(&d1_empty[b]);
				mbar_arrive(&a2_full[b]);
			}
		}
	}
	else if(warp < kMmaW)
	{
		// ================================================================ output
		const int ch = warp - kOutW0, k1 = lane;
		const int sb = ch >> 1, p = ch & 1;
		const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
		constexpr float osc = 1.0f / (float)(1 << kTcSpecExp);
		// this lane's offsets, read back only by itself
		uint32_t *otab = (uint32_t *)(base + LY::kOffOutTab) + ch * 1024 + lane;
		int tab_tcb = -1, tab_nrow = -1;
		for(int k = 0; k < nk; k++)
		{
			const int b = k & 1;
			if(!__all_sync(0xffffffffu, mbar_wait(&d2_full[b], (uint32_t)(k >> 1) & 1u, &fail_s)))
			{
				fail_s = 13;
				break;
			}
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			// channels k1 + 32 j, j in [0, 16) then [16, 32): 32 columns each
			float v[32];
			const uint32_t tcol = tmem + lane_base + (uint32_t)(256 * b + 128);
			tld32(tcol, v);
			tld_wait();
			const UnitRec &R = ring[k % kRing];
			const int row = R.row[sb][p];
			// channel c = k1 + 32 j: exp(2 pi i (ce D + post)), ce = c (upper
			// sideband) or c - nchan (lower), D = hi + lo (ce hi exact), stepped
			// by exp(2 pi i 32 D)
			const bool lsb = (R.flags & (sb == 0 ? kLsb0 : kLsb1)) != 0;
			const float fce = (float)(lsb ? k1 - nchan : k1);
			float th = fce * R.dhi[sb][p];
			th -= rintf(th);
			float turns = th + fmaf(fce, R.dlo[sb][p], R.post[sb][p]);
			turns -= rintf(turns);
			float qr, qi;
			__sincosf(6.283185307179586f * turns, &qi, &qr);
			qr *= osc;
			qi *= osc;
			float sr, si;
			__sincosf(6.283185307179586f * R.st32[sb][p], &si, &sr);
			const int tcb = R.tcb[sb];
			uint32_t *o = (uint32_t *)a.spec + R.spec[sb] + (int64_t)(row < 0 ? 0 : row) * tcb;
			if(row >= 0 && (tcb != tab_tcb || R.nrow[sb] != tab_nrow))
			{
				// channel c = k1 + 32 j sits at (c / tcb) nrow tcb + c % tcb
				tab_tcb = tcb;
				tab_nrow = R.nrow[sb];
				const uint32_t PT = (uint32_t)tab_nrow * (uint32_t)tcb;
				for(int j = 0; j < 32; j++)
				{
					const uint32_t c = (uint32_t)(k1 + 32 * j), blk = c / (uint32_t)tcb;
					otab[32 * j] = blk * PT + (c - blk * (uint32_t)tcb);
				}
			}
#pragma unroll
			for(int hh = 0; hh < 2; hh++)
			{
				if(hh == 1)
				{
					tld32(tcol + 32, v);
					tld_wait();
					asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
					__syncwarp();
					if(lane == 0)
						mbar_arrive(&d2_empty[b]);
				}
				if(row < 0)
					continue;
#pragma unroll
				for(int q = 0; q < 16; q++)
				{
					const int j = 16 * hh + q;
					const float xr = v[2 * q], xi = v[2 * q + 1];
					o[otab[32 * j]] = pack_spec(H16, xr * qr - xi * qi, xr * qi + xi * qr);
					const float nr = qr * sr - qi * si;
					qi = qr * si + qi * sr;
					qr = nr;
				}
			}
		}
	}
	else if(warp == kMmaW && lane == 0)
	{
		// ================================================================ MMA issuer
		// instruction descriptor: D F32 (bit 4), A and B F16, A MN-major (bit 15),
		// B K-major, N = 64 (bits 17-22: N >> 3), M = 128 (bits 24-28: M >> 4)
		const uint32_t idesc = (1u << 4) | (1u << 15) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
		const uint32_t aB1 = su32(base + kOffB1), aB2 = su32(base + kOffB2);
		auto mma2 = [&](int j) -> bool {
			const int b = j & 1, s = j % kNS;
			if(!mbar_wait(&a2_full[b], (uint32_t)(j >> 1) & 1u, &fail_s))
				return false;
			if(j >= 2 && !mbar_wait(&d2_empty[b], (uint32_t)((j >> 1) - 1) & 1u, &fail_s))
				return false;
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			const uint32_t bside = aB2 + ((ring[j % kRing].flags & kLsb0) ? kB2Bytes : 0);
			const uint32_t aA = su32(ops + s * kOpBytes);
			const uint32_t dcol = tmem + (uint32_t)(256 * b + 128);
#pragma unroll
			for(int ks = 0; ks < 8; ks++)
				mma_f16(dcol, desc_mn128(aA + ks * 4096), desc_k128(bside + (ks >> 2) * 8192 + (ks & 3) * 32), idesc,
				        ks > 0 ? 1u : 0u);
			commit_to(&d2_full[b]);
			commit_to(&op_empty[s]);
			return true;
		};
		bool ok = true;
		int k = 0;
		for(; k < nk && ok; k++)
		{
			const int b = k & 1, s = k % kNS;
			if(!mbar_wait(&op_full[s], (uint32_t)(k / kNS) & 1u, &fail_s) ||
			   (k >= 2 && !mbar_wait(&d1_empty[b], (uint32_t)((k >> 1) - 1) & 1u, &fail_s)))
			{
				fail_s = 14;
				ok = false;
				break;
			}
			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
			const uint32_t aA = su32(ops + s * kOpBytes);
#pragma unroll
			for(int sb = 0; sb < 2; sb++)
			{
				const uint32_t dcol = tmem + (uint32_t)(256 * b + 64 * sb);
#pragma unroll
				for(int ks = 0; ks < 4; ks++)
					mma_f16(dcol, desc_mn128(aA + sb * 16384 + ks * 4096), desc_k128(aB1 + ks * 32), idesc,
					        ks > 0 ? 1u : 0u);
			}
			commit_to(&d1_full[b]);
			if(k >= 1 && !mma2(k - 1))
			{
				fail_s = 15;
				ok = false;
			}
		}
		if(ok && k >= 1 && !mma2(k - 1))
			fail_s = 15;
		// every MMA issued by this thread has completed once this arrives
		commit_to(&mma_done);
		if(!mbar_wait(&mma_done, 0, &fail_s))
			fail_s = 16;
	}

	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	if(tid == 0)
	{
		// staged windows that no decode consumed (error path): wait (bounded) for
		// their copies before the shared memory goes away
		for(int k = stg_used_s; k < stg_issued_s; k++)
			mbar_wait(&stg_full[k % kNStg], (uint32_t)(k / kNStg) & 1u, &fail_s);
		if(fail_s && err)
			atomicExch(err, fail_s);
	}
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	if(warp == kMmaW)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)kTmemCols));
}

// ---------------------------------------------------------------- host side
// Constant tables in the kernel's shared-memory byte layout (values in
// double, rounded once to FP16), K-major with the 128-byte swizzle:
//   DFT-32: rows j = 2 k1 + part (out), K = part_in 32 + n1;
//   DFT-64 of the upper (k2 in [0, 32)) and lower (k2 in [32, 64)) sideband:
//          rows j = 2 k2' + part, K = part_in 64 + n2, two K halves of 64.
// A complex product (x_r + i x_i)(cos t - i sin t) is
//   re: x_r cos t + x_i sin t,  im: -x_r sin t + x_i cos t.
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
			put(o + kOffB1, 2 * k1, n1, c);
			put(o + kOffB1, 2 * k1, 32 + n1, sn);
			put(o + kOffB1, 2 * k1 + 1, n1, -sn);
			put(o + kOffB1, 2 * k1 + 1, 32 + n1, c);
		}
	for(int side = 0; side < 2; side++)
	{
		unsigned char *t = o + kOffB2 + side * kB2Bytes;
		for(int j = 0; j < 32; j++)
		{
			const int k2 = j + 32 * side;
			for(int n2 = 0; n2 < kN2; n2++)
			{
				const double ph = 2.0 * M_PI * (double)(n2 * k2 % kN2) / kN2;
				const double c = cos(ph), sn = sin(ph);
				// K = part_in 64 + n2: the real part's K half, then the imaginary part's
				put(t, 2 * j, n2, c);
				put(t + 8192, 2 * j, n2, sn);
				put(t, 2 * j + 1, n2, -sn);
				put(t + 8192, 2 * j + 1, n2, c);
			}
		}
	}
}

bool fstage_tc_eligible(int N, int order, bool any_lsb)
{
	return N == kN && (order == 1 || (order == 0 && !any_lsb));
}

cudaError_t launch_fstage_tc(const FKind &k, FsArgs a, int nsm, cudaStream_t stream)
{
	if(k.count <= 0 || a.T <= 0 || !k.tctab || !k.tcpairs || k.tcnpairs <= 0)
		return cudaSuccess;
	a.first = k.first;
	const int nunits = k.tcnpairs * a.T;
	int grid = nsm;
	if(grid > nunits)
		grid = nunits;
	auto go = [&](auto kern, size_t smem) {
		cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		kern<<<grid, kThreadsTc, smem, stream>>>(a, (const uint4 *)k.tctab, k.tcpairs, k.tcnpairs, nunits, a.err);
	};
	const bool h = a.h16 != 0;
	switch(k.tcbpt)
	{
	case 4: h ? go(k_fstage_tc<4, true>, TcLayout<4>::kSmem) : go(k_fstage_tc<4, false>, TcLayout<4>::kSmem); break;
	case 8: h ? go(k_fstage_tc<8, true>, TcLayout<8>::kSmem) : go(k_fstage_tc<8, false>, TcLayout<8>::kSmem); break;
	case 16: h ? go(k_fstage_tc<16, true>, TcLayout<16>::kSmem) : go(k_fstage_tc<16, false>, TcLayout<16>::kSmem); break;
	case 32: h ? go(k_fstage_tc<32, true>, TcLayout<32>::kSmem) : go(k_fstage_tc<32, false>, TcLayout<32>::kSmem); break;
	case 64: h ? go(k_fstage_tc<64, true>, TcLayout<64>::kSmem) : go(k_fstage_tc<64, false>, TcLayout<64>::kSmem); break;
	default: break;
	}
	return cudaGetLastError();
}

}  // namespace fxb
