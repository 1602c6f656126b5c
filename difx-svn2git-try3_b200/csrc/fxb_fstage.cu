// F stage (Mode::process, mpifxcorr/src/mode.cpp:845-1308) for sm_100a.
//
// One CTA per (station, subband, chunk of FFTs); a subband's one or two
// polarisation bands are transformed together.  The FFT length is a template
// parameter, so the pass schedule and every shared-memory index fold to
// constants.  Each thread owns KB radix-8 butterflies of every pass of one
// FFT ("slot"): an FFT of N points takes N / (8 KB) threads, and a CTA runs
// several slots side by side when N is small.  Per FFT a thread
//   1. decodes its 8 KB samples x[b + r N/8] straight from the VDIF words in
//      global memory (2-bit / 8-bit levels of format_vdif.c:74-149; samples of
//      invalid frames and, for 8-bit 2/4-channel streams, every sample after
//      the first blanked one, read as zero: format_vdif.c:1879-1922),
//   2. multiplies them by the fringe rotator exp(-2 pi i phi(n)) of the order
//      in use (mode.cpp:906-1051; phi reduced to [-1/2, 1/2) turns in FP64 at
//      the FFT start, per sample in FP32),
//   3. runs the first radix-8 pass of a Stockham autosort FFT in registers
//      and exchanges through padded shared memory for the remaining passes
//      (two buffers used alternately: one barrier per exchange),
//   4. in the last pass selects the sideband (USB bins 0..nchan-1, LSB
//      nchan..2nchan-1, order-0 LSB the conjugate mirror), applies the
//      fractional-sample rotator exp(+2 pi i f_c fse) (mode.cpp:1053-1097,
//      1279-1286) and the post-F fringe phase of order 0 (mode.cpp:1061-1070),
//      and stores its channels to the spectra [t][row][chan].
//
// The FFT is FP32.  Two output forms:
//   out 0: spectra as float2 [t][row][chan] (the plain FP32 form);
//   out 1: spectra of the tensor-core forms, half2 or bf16x2 (re, im) of
//          X 2^-kTcSpecExp in the blocked layout the tensor-core XMAC reads
//          (one rounding per value, for the kinds the tensor-core FFT of
//          fxb_fstage_tc.cu does not cover).
//
// Twiddles come from a per-length table laid out [pass][r - 1][p] (entry
// w_N^(r p s) for pass stride s), so that the twiddle loads of a warp are
// coalesced (first pass) or broadcasts (later passes).

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <type_traits>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

namespace {

// padded index of 8-byte element i: every exchange of the pass schedule
// below is free of bank conflicts, and runs of 8 starting at multiples of 8
// stay contiguous and 16-byte aligned (the first pass stores them as pairs)
__host__ __device__ constexpr int xpad(int i) { return i + 2 * (i >> 4); }

// Compile-time shape of the F stage for FFT length 2^LOGN.
template <int LOGN>
struct FShape {
	static constexpr int N = 1 << LOGN;
	static constexpr int KB = N <= 2048 ? 1 : (N <= 8192 ? 2 : 4);
	static constexpr int TPF = N / (8 * KB);                 // threads per FFT
	static constexpr int NT = TPF >= 256 ? TPF : 256;        // threads per CTA
	static constexpr int FPC = NT / TPF;                     // FFTs side by side
	static constexpr int PADN = xpad(N);
	static constexpr int NMID = (LOGN % 3 == 0) ? LOGN / 3 - 2 : LOGN / 3 - 1;
	static constexpr int RL = (LOGN % 3 == 0) ? 8 : (1 << (LOGN % 3));
	// 8192 points: two butterflies per thread in 512-thread CTAs at 64 registers
	// (two CTAs per SM) run 37 % faster than four per thread at 128 registers
	static constexpr int MINB = KB == 1 ? 3 : (NT == 256 || KB == 2 ? 2 : 1);
};

// offset of the twiddles of radix-8 pass `pass` (stride 8^pass) in the table
__host__ __device__ constexpr int tw_offset(int N, int pass)
{
	int o = 0, n8 = N / 8;
	for(int i = 0; i < pass; i++)
	{
		o += 7 * n8;
		n8 /= 8;
	}
	return o;
}

// padded index of element i + S r (i >= 0): for S a multiple of 16 the
// padding of i + S r is that of i plus r S / 8, a constant offset per r.
// Used for FFTs of 8192 points and more (FAST); shorter lengths keep the
// plain form, whose register allocation measured better.
template <int S, bool FAST>
__device__ __forceinline__ int st_index(int i, int r)
{
	if constexpr(FAST && S % 16 == 0)
		return xpad(i) + r * xpad(S);
	else
		return xpad(i + S * r);
}

// ---- lane values: FP32 complex
struct cf { float x, y; };

__device__ __forceinline__ cf add(cf a, cf b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cf sub(cf a, cf b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cf add_mi(cf a, cf b) { return {a.x + b.y, a.y - b.x}; }   // a - i b
__device__ __forceinline__ cf add_pi(cf a, cf b) { return {a.x - b.y, a.y + b.x}; }   // a + i b
__device__ __forceinline__ cf rot45(cf a)                                               // a (1 - i) / sqrt2
{
	const float r = 0.70710678118654752440f;
	return {(a.x + a.y) * r, (a.y - a.x) * r};
}
__device__ __forceinline__ cf twid(cf a, float2 w) { return {a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x}; }

__device__ __forceinline__ float2 ldtw(const float2 *t, int i) { return __ldg(t + i); }
// 8-byte shared-memory element <-> lane value
template <typename C> __device__ __forceinline__ C lds(const uint2 *p);
template <> __device__ __forceinline__ cf lds<cf>(const uint2 *p)
{
	const float2 v = *(const float2 *)p;
	return {v.x, v.y};
}
__device__ __forceinline__ uint2 bits(cf v) { return make_uint2(__float_as_uint(v.x), __float_as_uint(v.y)); }
template <typename C> __device__ __forceinline__ void sts(uint2 *p, C v) { *p = bits(v); }
template <typename C> __device__ __forceinline__ void sts2(uint2 *p, C a, C b)
{
	const uint2 u = bits(a), w = bits(b);
	*(uint4 *)p = make_uint4(u.x, u.y, w.x, w.y);
}

// forward DFTs in place (w = exp(-2 pi i / R))
template <typename C>
__device__ __forceinline__ void dft8(C *x)
{
	const C a0 = add(x[0], x[4]), d0 = sub(x[0], x[4]);
	const C a1 = add(x[1], x[5]), d1 = sub(x[1], x[5]);
	const C a2 = add(x[2], x[6]), d2 = sub(x[2], x[6]);
	const C a3 = add(x[3], x[7]), d3 = sub(x[3], x[7]);
	const C b0 = add(a0, a2), b2 = sub(a0, a2), b1 = add(a1, a3), b3 = sub(a1, a3);
	x[0] = add(b0, b1);
	x[4] = sub(b0, b1);
	x[2] = add_mi(b2, b3);
	x[6] = add_pi(b2, b3);
	// odd bins: DFT4 of d_k w^k, with d1 w + d3 w^3 = (d1 - i d3) w and d1 w - d3 w^3 = (d1 + i d3) w
	const C f0 = add_mi(d0, d2), f2 = add_pi(d0, d2);
	const C f1 = rot45(add_mi(d1, d3)), f3 = rot45(add_pi(d1, d3));
	x[1] = add(f0, f1);
	x[5] = sub(f0, f1);
	x[3] = add_mi(f2, f3);
	x[7] = add_pi(f2, f3);
}

template <typename C>
__device__ __forceinline__ void dft4(C *x)
{
	const C b0 = add(x[0], x[2]), b2 = sub(x[0], x[2]), b1 = add(x[1], x[3]), b3 = sub(x[1], x[3]);
	x[0] = add(b0, b1);
	x[2] = sub(b0, b1);
	x[1] = add_mi(b2, b3);
	x[3] = add_pi(b2, b3);
}

template <typename C>
__device__ __forceinline__ void dft2(C *x)
{
	const C a = x[0], b = x[1];
	x[0] = add(a, b);
	x[1] = sub(a, b);
}

template <int R, typename C>
__device__ __forceinline__ void dftR(C *x)
{
	if constexpr(R == 8)
		dft8(x);
	else if constexpr(R == 4)
		dft4(x);
	else
		dft2(x);
}

// 2-bit code -> {-HiMag, -1, +1, +HiMag} (format_vdif.c:78): sign from bit 1,
// magnitude HiMag for codes 0 and 3
__host__ __device__ inline float level2(uint32_t code)
{
	const float mag = ((code ^ (code >> 1)) & 1u) ? 1.0f : 3.3359f;
	return (code & 2u) ? mag : -mag;
}

__device__ __forceinline__ float frac_centered(double x) { return (float)(x - rint(x)); }

// one spectral value of the tensor-core forms: (re, im) as half2 or bf16x2
__device__ __forceinline__ uint32_t pack_spec(bool h16, float re, float im)
{
	if(h16)
	{
		const __half2 h = __floats2half2_rn(re, im);
		return *(const uint32_t *)&h;
	}
	const __nv_bfloat162 b = __floats2bfloat162_rn(re, im);
	return *(const uint32_t *)&b;
}

// CTAs per SM the register budget is sized for
template <int LOGN>
constexpr int fstage_minb()
{
	return FShape<LOGN>::MINB;
}

constexpr int kMaxTQ = 4;         // FFT iterations per CTA at most

// Constants of one FFT, computed once per CTA (one warp per FFT).
struct FftConst {
	float P0, alpha, beta, gamma, eps;   // fringe phase (turns): start and per-sample terms
	float stc, sts;                      // order 1: rotator step over N/8 samples, exp(-2 pi i alpha N/8)
	float dhi[2], dlo[2];                // fractional-sample turns per channel of each band (split_turns)
	float postf;                         // order-0 post-F turns
	uint32_t fa, so;                     // first frame of the window, window start within it
	uint32_t fmask;                      // validity of the window's frames (bit k: frame fa + k)
	int32_t stuck;                       // samples [stuck, N) read as zero
	int32_t flags;                       // 1: valid FFT, 2: fmask covers the window,
	                                     // 4: a valid frame of the window blanks one of the item's bands,
	                                     // 8: the two bands take the same output rotation
};

// One middle radix-8 pass (stride s = 2^LOGS, m = N / (8 s)) over the
// thread's KB butterflies: x_r = X[q + s (p + r m)], y = DFT8(x),
// Y[q + s (8 p + r)] = y_r w_N^(r p s).  With two buffers each butterfly
// reads, transforms and writes on its own; with one buffer all reads of the
// pass come before any write.
template <typename C, int NV, int LOGN, int LOGS, typename TW, class Team>
__device__ __forceinline__ void mid_pass(int &wb, uint2 *side0, uint2 *side1, int pp, int bt, const TW *twp,
                                         const Team &tm)
{
	using SH = FShape<LOGN>;
	constexpr int N = SH::N, KB = SH::KB, TPF = SH::TPF, PADN = SH::PADN;
	constexpr int s = 1 << LOGS;
	constexpr int m = N >> (LOGS + 3);
	constexpr int np = N / (8 * s);
	const uint2 *src = wb ? side1 : side0;
	wb ^= 1;
	uint2 *dst = wb ? side1 : side0;
	C x[KB][NV][8];
#pragma unroll
	for(int k = 0; k < KB; k++)
	{
		const int b = bt + k * TPF;
		const int q = b & (s - 1), p8 = b >> LOGS;
#pragma unroll
		for(int j = 0; j < NV; j++)
		{
#pragma unroll
			for(int r = 0; r < 8; r++)
			{
				// for N >= 128 the stride s m = N/8 is a multiple of 16, so the
				// padding of point r is a constant offset from that of point 0
				if constexpr(N >= 128)
					x[k][j][r] = lds<C>(src + j * PADN + xpad(q + s * p8) + r * xpad(s * m));
				else
					x[k][j][r] = lds<C>(src + j * PADN + xpad(q + s * (p8 + r * m)));
			}
			dft8(x[k][j]);
		}
#pragma unroll
		for(int r = 1; r < 8; r++)
		{
			const TW w = ldtw(twp, (r - 1) * np + p8);
#pragma unroll
			for(int j = 0; j < NV; j++)
				x[k][j][r] = twid(x[k][j][r], w);
		}
		if(pp)
		{
#pragma unroll
			for(int j = 0; j < NV; j++)
#pragma unroll
				for(int r = 0; r < 8; r++)
					sts(dst + j * PADN + st_index<s, (N >= 8192)>(q + s * 8 * p8, r), x[k][j][r]);
		}
	}
	if(!pp)
	{
		tm.sync();
#pragma unroll
		for(int k = 0; k < KB; k++)
		{
			const int b = bt + k * TPF;
			const int q = b & (s - 1), p8 = b >> LOGS;
#pragma unroll
			for(int j = 0; j < NV; j++)
#pragma unroll
				for(int r = 0; r < 8; r++)
					sts(dst + j * PADN + st_index<s, (N >= 8192)>(q + s * 8 * p8, r), x[k][j][r]);
		}
	}
	tm.sync();
}

template <typename C, int NV, int LOGN, int PS>
struct MidPasses {
	template <typename TW, class Team>
	__device__ static __forceinline__ void run(int &wb, uint2 *side0, uint2 *side1, int pp, int bt, const TW *tw,
	                                           const Team &tm)
	{
		if constexpr(PS < FShape<LOGN>::NMID)
		{
			mid_pass<C, NV, LOGN, 3 * (PS + 1)>(wb, side0, side1, pp, bt, tw + tw_offset(1 << LOGN, PS + 1), tm);
			MidPasses<C, NV, LOGN, PS + 1>::run(wb, side0, side1, pp, bt, tw, tm);
		}
	}
};

}  // namespace

// The threads that run one work unit: the whole CTA (barrier 0), or one
// half of a persistent CTA (named barrier 1 + half, 256 threads).
struct CtaTeam {
	__device__ __forceinline__ int tid() const { return threadIdx.x; }
	__device__ __forceinline__ int nt() const { return blockDim.x; }
	__device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct HalfTeam {
	int h;
	__device__ __forceinline__ int tid() const { return threadIdx.x & 255; }
	__device__ __forceinline__ int nt() const { return 256; }
	__device__ __forceinline__ void sync() const { asm volatile("bar.sync %0, 256;\n" ::"r"(1 + h) : "memory"); }
};

// Level tables of the decode: 8-bit levels (b - 128) / 3.3 computed in double
// and rounded to float (format_vdif.c:122), and two adjacent 2-bit bands ->
// (band0, band1) levels.
template <class Team>
__device__ __forceinline__ void fstage_luts(const Team &tm, bool eight, float *lut8, float2 *lut4)
{
	if(eight)
		for(int i = tm.tid(); i < 256; i += tm.nt())
			lut8[i] = (float)((i - 128) / 3.3);
	if(tm.tid() < 16)
		lut4[tm.tid()] = make_float2(level2(tm.tid() & 3u), level2(tm.tid() >> 2u));
}

// One work unit of the F stage: FFT times [tchunk tq FPC, +tq FPC) of work
// item gidx (an FGroup), run by the team's FShape<LOGN>::NT threads with the
// level tables already in shared memory, fsm the unit's exchange buffers
// (two when pp) and fcs room for tq FPC FFT constants.
// NV: bands of the item (values per point); TCO: tensor-core spectra out;
// VAR 1: raw INTERLACEDVDIF reads (each band read from its thread's frame);
// VAR 2: complex sampling (nchan-point complex FFT: every bin a channel of
// the upper sideband, or bin 0 and the conjugated mirror of the rest for the
// lower sideband, mode.cpp:1182-1234).
template <int NV, int LOGN, bool TCO, int VAR, class Team>
__device__ __forceinline__ void fstage_unit(const FsArgs &a, const int gidx, const int tchunk, const int tq, const int pp,
                                            const float2 *tw, uint2 *fsm, const float *lut8, const float2 *lut4,
                                            FftConst *fcs, const Team &tm)
{
	using SH = FShape<LOGN>;
	using C = cf;
	using TW = float2;
	constexpr int N = SH::N, KB = SH::KB, TPF = SH::TPF, FPC = SH::FPC, PADN = SH::PADN, RL = SH::RL;
	const FGroup g = a.groups[gidx];
	const DevStation *Sp = a.st + g.station;
	constexpr bool MUX = VAR == 1, CPLX = VAR == 2;
	constexpr int nchan = CPLX ? N : N / 2;
	const uint32_t fs = (uint32_t)Sp->framesamples;
	const int nbits = Sp->nbits;
	// raw INTERLACEDVDIF reads: band b's samples are those of its thread's
	// frame, found through the frame-slot table (one band per frame)
	constexpr bool muxraw = MUX;
	const int32_t *mslot = muxraw ? a.sub[g.station].mux_slot : nullptr;
	const int64_t mk0 = muxraw ? a.sub[g.station].mux_k0 : 0;
	const int mnthr = Sp->nthr, minfb = Sp->inframebytes;
	// complex samples: real then imaginary field of nbits per band and time
	constexpr uint32_t cpl = CPLX ? 2u : 1u;
	const uint32_t bpt = muxraw ? (uint32_t)nbits : (uint32_t)(Sp->nband * nbits) * cpl;
	const int header = Sp->header, framebytes = Sp->framebytes, asl = Sp->asl;
	const double bw = Sp->bw;
	const uint8_t *buf = a.sub[g.station].buf;
	const int slot = tm.tid() / TPF, bt = tm.tid() - slot * TPF;
	uint2 *const side0 = fsm + (size_t)slot * NV * PADN;
	uint2 *const side1 = pp ? side0 + (size_t)FPC * NV * PADN : side0;
	const uint8_t *vrow = a.valid + (int64_t)g.station * a.valid_stride;
	const int64_t spec_off = a.plans[g.freq].spec_off;
	const int prow = a.plans[g.freq].nrow;
	// tensor-core form: spectra blocked [t][block][row][tcb] (tcb channels per block)
	const uint32_t tcb = (uint32_t)a.plans[g.freq].tcb, tnblk = (uint32_t)a.plans[g.freq].tnblk;
	const uint32_t tcb_magic = tcb ? 0xFFFFFFFFu / tcb + 1u : 0u;    // c / tcb = umulhi(c, magic) for c < 2^16
	const bool lsb = g.lsb != 0;
	const double lo = g.lofreq;
	const float ph0 = g.phase[0], ph1 = g.phase[1];     // phase-offset rotation of each band (turns)
	const int row0 = g.row[0], row1 = g.row[1];
	const uint32_t boff0 = muxraw ? 0u : (uint32_t)(g.band[0] * nbits) * cpl,
	               boff1 = muxraw ? 0u : (uint32_t)(g.band[1] * nbits) * cpl;
	const bool oneword = !muxraw && bpt <= 32;       // all bands of a sample time in one 32-bit word
	const bool pair4 = !CPLX && NV == 2 && nbits == 2 && oneword && boff1 == boff0 + 2;
	const int order = a.order;
	constexpr float osc = 1.0f / (float)(1 << kTcSpecExp);
	const bool h16 = a.h16 != 0;

	const int t0 = tchunk * tq * FPC;
	const int nit = min(tq, (a.T - t0 + FPC - 1) / FPC);
	// ---- constants of the unit's FFTs (FFT f is time t0 + f), one thread per FFT
	{
		const int nfc = nit * FPC;
		for(int f = tm.tid(); f < nfc; f += tm.nt())
		{
			const int t = t0 + f;
			FftConst c;
			c.P0 = c.alpha = c.beta = c.gamma = c.eps = c.postf = 0.0f;
			c.dhi[0] = c.dhi[1] = c.dlo[0] = c.dlo[1] = 0.0f;
			c.stc = 1.0f;
			c.sts = 0.0f;
			c.fa = c.so = c.fmask = 0u;
			c.stuck = 0;
			c.flags = 0;
			if(t < a.T)
			{
				const FftParam *pq = a.params + (int64_t)g.station * a.T + t;
				if(pq->status == kFftOk)
				{
					c.flags = 1;
					const uint32_t g0 = (uint32_t)pq->nearest;
					c.fa = g0 / fs;
					c.so = g0 - c.fa * fs;
					c.stuck = pq->stuck;
					const double invN = 1.0 / N;
					const int idl = pq->integerdelay;
					const double fraclo = a.fraclo ? (lo - (int)lo) * (double)idl : 0.0;
					// LO offset: seconds since the job start of the FFT's first
					// sample (mode.cpp:686-694; the scan starts with the job) and
					// the offset's turns per sample
					const double walls = (double)a.sub[g.station].subsec + a.sub[g.station].subns / 1.0e9 +
					                     (double)t * N * Sp->sampletime / 1.0e6;
					const double low = g.corr ? looff_wall_turns(g.looff, walls) : 0.0;
					const double los = -g.looff * Sp->sampletime / 1.0e6;
					if(order == 1)
					{
						c.P0 = frac_centered(lo * pq->b + fraclo + low);
						c.alpha = (float)(lo * pq->a * invN + los);
						// each thread's samples are N/8 apart: one step phasor per FFT
						const double st = (double)c.alpha * (double)(N / 8);
						double ss, sc;
						sincospi(-2.0 * (st - rint(st)), &ss, &sc);
						c.stc = (float)sc;
						c.sts = (float)ss;
					}
					else if(order == 2)
					{
						const double pa = pq->a, pb = pq->b;
						const double X1 = (double)asl * invN;
						c.P0 = frac_centered(lo * pq->c + fraclo + low);
						c.alpha = (float)(lo * (pb + pa * X1) * invN + los);
						c.beta = (float)(lo * 2.0 * pa * X1 * invN);
						c.gamma = (float)(lo * pb * asl * invN + los * asl);
						c.eps = (float)(lo * pa * X1 * X1);
					}
					// per band: fse - clock offset (mode.cpp:1053-1059, 1099-1106)
					split_turns(bw * (1.0 / nchan) * ((double)pq->fse - g.clk[0]), c.dhi[0], c.dlo[0]);
					split_turns(bw * (1.0 / nchan) * ((double)pq->fse - g.clk[1]), c.dhi[1], c.dlo[1]);
					if(order == 0)
					{
						double pr = (pq->averagedelay - idl) * lo;
						if(a.fraclo)
							pr += idl * (lo - (int)lo);
						pr -= walls * g.looff;
						c.postf = -(float)(pr - (int)pr);
					}
				}
			}
			// validity of the window's frames, one bit per frame relative to fa
			const uint32_t nwf = (c.so + (uint32_t)N - 1) / fs + 1;
			if(c.flags & 1)
			{
				const uint32_t nm = nwf < 32u ? nwf : 32u;
				for(uint32_t k = 0; k < nm; k++)
				{
					const int64_t fr = (int64_t)c.fa + k;
					// complex data: the unpack's first frame is checked for fill
					// pattern only (mark5_stream_unpacker.c:189)
					const uint8_t *vsrc =
					    (CPLX && k == 0 && a.fillok) ? a.fillok + (int64_t)g.station * a.valid_stride : vrow;
					if(fr < a.valid_stride && vsrc[fr] != 0)
						c.fmask |= 1u << k;
				}
			}
			if(nwf <= 32)
				c.flags |= 2;
			if(c.dhi[0] == c.dhi[1] && c.dlo[0] == c.dlo[1] && g.phase[0] == g.phase[1])
				c.flags |= 8;
			if(a.bandok)
			{
				// EDV4-blanked bands (INTERLACEDVDIF): the slow decode path below
				const uint32_t need = (1u << g.band[0]) | (g.band[1] >= 0 ? 1u << g.band[1] : 0u);
				bool part = false;
				for(uint32_t k = 0; (c.flags & 1) && k < nwf && !part; k++)
				{
					const int64_t fk = (int64_t)c.fa + k;
					part = fk < a.valid_stride && vrow[fk] != 0 &&
					       (a.bandok[(int64_t)g.station * a.valid_stride + fk] & need) != need;
				}
				if(part)
					c.flags |= 4;
			}
			fcs[f] = c;
		}
		tm.sync();
	}
	int wb = 0;
	for(int it = 0; it < nit; it++)
	{
		const int t = t0 + it * FPC + slot;
		const bool tok = t < a.T;
		// ---- per-FFT constants
		const FftConst &fc = fcs[it * FPC + slot];
		const bool active = (fc.flags & 1) != 0;
		const uint32_t fa = fc.fa, so = fc.so, fmask = fc.fmask;
		const int stuck = fc.stuck;
		const float P0 = fc.P0, alpha = fc.alpha, beta = fc.beta, gamma = fc.gamma, eps = fc.eps;
		const float stc = fc.stc, sts = fc.sts;
		const float dhi0 = fc.dhi[0], dlo0 = fc.dlo[0], dhi1 = fc.dhi[1], dlo1 = fc.dlo[1], postf = fc.postf;
		const bool narrow = (fc.flags & 2) != 0;
		const bool same = (fc.flags & 8) != 0;
		const bool blank = (fc.flags & 4) != 0;
		// ---- 1-3. decode, fringe-rotate and run the first radix-8 pass (s = 1:
		// butterfly b, twiddle w_N^(r b)), one butterfly at a time
		{
			uint2 *dst = wb ? side1 : side0;
			if(!pp)
				tm.sync();                    // the single buffer has been read by the last FFT
#pragma unroll
			for(int k = 0; k < KB; k++)
			{
				const int b = bt + k * TPF;
				const uint32_t xs = so + (uint32_t)b;
				uint32_t kf = xs / fs, tin = xs - kf * fs;
				const uint8_t *fp = buf + ((int64_t)fa + kf) * framebytes + header;
				// phase A: frame tracking and every word load of the 8 samples
				// (nothing waits on a load before all are issued)
				uint32_t raw0[8], raw1[8], pk[8];
#pragma unroll
				for(int r = 0; r < 8; r++)
				{
					const int n = b + r * (N / 8);
					bool ok;
					if(narrow)
						ok = (fmask >> kf) & 1u;
					else
					{
						const int64_t fr = (int64_t)fa + kf;
						ok = active && fr < a.valid_stride && vrow[fr] != 0;
					}
					ok = ok && n < stuck;
					const uint32_t bit0 = tin * bpt + boff0, bit1 = tin * bpt + boff1;
					if(muxraw)
					{
						// valid frames of raw reads are complete slots: every thread is there
						const int32_t *slr = mslot + (mk0 + (int64_t)fa + kf) * mnthr;
						const int i0 = ok ? __ldg(slr + g.band[0]) : -1;
						const int i1 = (ok && NV == 2) ? __ldg(slr + g.band[1]) : -1;
						raw0[r] = i0 >= 0 ? __ldg((const uint32_t *)(buf + (int64_t)i0 * minfb + 32) + (bit0 >> 5)) : 0u;
						raw1[r] = i1 >= 0 ? __ldg((const uint32_t *)(buf + (int64_t)i1 * minfb + 32) + (bit1 >> 5)) : 0u;
					}
					else
					{
						const uint32_t *wp = (const uint32_t *)fp;
						raw0[r] = ok ? __ldg(wp + (bit0 >> 5)) : 0u;
						raw1[r] = (ok && !oneword && NV == 2) ? __ldg(wp + (bit1 >> 5)) : 0u;
					}
					pk[r] = (bit0 & 31u) | ((bit1 & 31u) << 8) | ((uint32_t)ok << 16);
					if(r < 7)
					{
						tin += (uint32_t)(N / 8);
						while(tin >= fs)
						{
							tin -= fs;
							kf++;
							fp += framebytes;
						}
					}
				}
				// phase B: levels, fringe rotation (order 1: the rotator of sample b,
				// then one complex step per N/8 samples)
				float rc = 1.0f, rs = 0.0f;
				if(order == 1)
				{
					float ph0 = P0 + (float)b * alpha;
					ph0 -= rintf(ph0);
					__sincosf(-6.283185307179586f * ph0, &rs, &rc);
				}
				C x[NV][8];
#pragma unroll
				for(int r = 0; r < 8; r++)
				{
					const int n = b + r * (N / 8);
					float v0 = 0.0f, v1 = 0.0f, u0 = 0.0f, u1 = 0.0f;     // u: imaginary parts (complex sampling)
					if((pk[r] >> 16) & 1u)
					{
						const uint32_t w0 = raw0[r] >> (pk[r] & 31u);
						if(pair4)
						{
							const float2 l = lut4[w0 & 15u];
							v0 = l.x;
							v1 = l.y;
						}
						else
						{
							v0 = nbits == 2 ? level2(w0 & 3u) : lut8[w0 & 255u];
							if constexpr(CPLX)
								u0 = nbits == 2 ? level2((w0 >> 2) & 3u) : lut8[(w0 >> 8) & 255u];
							if(NV == 2)
							{
								const uint32_t w1 = (oneword ? raw0[r] : raw1[r]) >> ((pk[r] >> 8) & 31u);
								v1 = nbits == 2 ? level2(w1 & 3u) : lut8[w1 & 255u];
								if constexpr(CPLX)
									u1 = nbits == 2 ? level2((w1 >> 2) & 3u) : lut8[(w1 >> 8) & 255u];
							}
						}
						if(blank)
						{
							// bands of this sample's frame blanked by its EDV4 validity mask
							// (blank_vdif_EDV4, format_vdif.c:4699-4780)
							const uint32_t bo = a.bandok[(int64_t)g.station * a.valid_stride + fa + (so + (uint32_t)n) / fs];
							if(!((bo >> g.band[0]) & 1u))
								v0 = u0 = 0.0f;
							if(g.band[1] >= 0 && !((bo >> g.band[1]) & 1u))
								v1 = u1 = 0.0f;
						}
					}
					float sn = 0.0f, cs = 1.0f;
					if(order == 1)
					{
						cs = rc;
						sn = rs;
						const float nc = rc * stc - rs * sts;
						rs = rc * sts + rs * stc;
						rc = nc;
					}
					else if(order == 2)
					{
						const int kk = n / asl, jj = n - kk * asl;
						float ph = P0 + (float)jj * alpha + (float)(kk * jj) * beta + (float)kk * gamma +
						           (float)(kk * kk) * eps;
						ph -= rintf(ph);
						__sincosf(-6.283185307179586f * ph, &sn, &cs);
					}
					if constexpr(CPLX)
					{
						x[0][r] = cf{v0 * cs - u0 * sn, v0 * sn + u0 * cs};
						if constexpr(NV == 2)
							x[1][r] = cf{v1 * cs - u1 * sn, v1 * sn + u1 * cs};
					}
					else
					{
						x[0][r] = cf{v0 * cs, v0 * sn};
						if constexpr(NV == 2)
							x[1][r] = cf{v1 * cs, v1 * sn};
					}
				}
#pragma unroll
				for(int j = 0; j < NV; j++)
					dft8(x[j]);
#pragma unroll
				for(int r = 1; r < 8; r++)
				{
					const TW w = ldtw(tw, (r - 1) * (N / 8) + b);
#pragma unroll
					for(int j = 0; j < NV; j++)
						x[j][r] = twid(x[j][r], w);
				}
				const int o = xpad(8 * b);
#pragma unroll
				for(int j = 0; j < NV; j++)
				{
					uint2 *q = dst + j * PADN + o;
					sts2(q, x[j][0], x[j][1]);
					sts2(q + 2, x[j][2], x[j][3]);
					sts2(q + 4, x[j][4], x[j][5]);
					sts2(q + 6, x[j][6], x[j][7]);
				}
			}
			tm.sync();
		}
		// ---- middle radix-8 passes through shared memory
		MidPasses<C, NV, LOGN, 0>::run(wb, side0, side1, pp, bt, tw, tm);
		// ---- 4. last pass, sideband selection, fractional-sample rotation, output
		{
			constexpr int sL = N / RL;
			constexpr int J = (KB * 8) / RL;
			const uint2 *src = wb ? side1 : side0;
			wb ^= 1;
			const int64_t obase = spec_off + (int64_t)t * prow * nchan;
#pragma unroll
			for(int jj = 0; jj < J; jj++)
			{
				const int q = bt + jj * TPF;
				C y[NV][RL];
#pragma unroll
				for(int j = 0; j < NV; j++)
				{
#pragma unroll
					for(int r = 0; r < RL; r++)
						y[j][r] = lds<C>(src + j * PADN + st_index<sL, (N >= 8192)>(q, r));
					dftR<RL>(y[j]);
				}
				if(!tok)
					continue;
#pragma unroll
				for(int r = 0; r < RL; r++)
				{
					const int k = q + sL * r;
					int c, ce;
					float cj = 1.0f;
					if constexpr(CPLX)
					{
						// every bin is a channel; the lower sideband keeps bin 0 and
						// mirrors and conjugates the rest (mode.cpp:1217-1226)
						if(!lsb)
						{
							c = k;
							ce = k;
						}
						else
						{
							c = k == 0 ? 0 : N - k;
							ce = c - nchan;
							cj = k == 0 ? 1.0f : -1.0f;
						}
					}
					else if(!lsb)
					{
						if(r >= RL / 2)
							continue;                  // bins >= nchan
						c = k;
						ce = k;
					}
					else if(order != 0)
					{
						if(r < RL / 2)
							continue;
						c = k - nchan;
						ce = c - nchan;
					}
					else
					{
						if(!(k >= 1 && k <= nchan))
							continue;
						c = nchan - k;
						ce = c - nchan;
						cj = -1.0f;
					}
					// fractional-sample (and order-0 fringe) rotation of band 0 and,
					// where its clock or phase offset differs, of band 1
					const float fce = (float)ce;
					float t0h = fce * dhi0;             // exact (split_turns)
					t0h -= rintf(t0h);
					float turns = t0h + fmaf(fce, dlo0, postf + ph0);
					turns -= rintf(turns);
					float sn, cs;
					__sincosf(6.283185307179586f * turns, &sn, &cs);
					float sn1 = sn, cs1 = cs;
					if(NV == 2 && !same)
					{
						float t1h = fce * dhi1;
						t1h -= rintf(t1h);
						float turns1 = t1h + fmaf(fce, dlo1, postf + ph1);
						turns1 -= rintf(turns1);
						__sincosf(6.283185307179586f * turns1, &sn1, &cs1);
					}
					if constexpr(TCO)
					{
						uint32_t *o;
						int64_t rstride;
						if(tcb)
						{
							const uint32_t blk = __umulhi((uint32_t)c, tcb_magic), cl = (uint32_t)c - blk * tcb;
							o = (uint32_t *)a.spec + spec_off + (((int64_t)t * tnblk + blk) * prow) * tcb + cl;
							rstride = tcb;
						}
						else
						{
							o = (uint32_t *)a.spec + obase + c;
							rstride = nchan;
						}
#pragma unroll
						for(int j = 0; j < NV; j++)
						{
							const int rw = j == 0 ? row0 : row1;
							const float ocs = (j == 0 ? cs : cs1) * osc, osn = (j == 0 ? sn : sn1) * osc;
							if(rw >= 0)
							{
								const float xr = y[j][r].x, xi = cj * y[j][r].y;
								o[(int64_t)rw * rstride] = pack_spec(h16, xr * ocs - xi * osn, xr * osn + xi * ocs);
							}
						}
					}
					else
					{
						float2 *o = (float2 *)a.spec + obase + c;
#pragma unroll
						for(int j = 0; j < NV; j++)
						{
							const int rw = j == 0 ? row0 : row1;
							const float ocs = j == 0 ? cs : cs1, osn = j == 0 ? sn : sn1;
							if(rw >= 0)
							{
								const float xr = y[j][r].x, xi = cj * y[j][r].y;
								o[(int64_t)rw * nchan] = make_float2(xr * ocs - xi * osn, xr * osn + xi * ocs);
							}
						}
					}
				}
			}
		}
	}
}

// One CTA per work unit.  grid: (time chunks, items), or (items, time chunks)
// when the stations of a subband should run side by side (blocked
// tensor-core spectra).
template <int NV, int LOGN, bool TCO, int VAR>
__global__ void __launch_bounds__(FShape<LOGN>::NT, fstage_minb<LOGN>()) k_fstage(const FsArgs a)
{
	extern __shared__ __align__(16) uint2 fsm[];
	__shared__ float lut8[256];
	__shared__ float2 lut4[16];
	__shared__ FftConst fcs[kMaxTQ * FShape<LOGN>::FPC];
	const CtaTeam tm;
	const int item = a.items_fast ? blockIdx.x : blockIdx.y;
	const int tchunk = a.items_fast ? blockIdx.y : blockIdx.x;
	fstage_luts(tm, a.st[a.groups[a.first + item].station].nbits == 8, lut8, lut4);
	tm.sync();
	fstage_unit<NV, LOGN, TCO, VAR>(a, a.first + item, tchunk, a.tq, a.pp, (const float2 *)a.tw, fsm, lut8, lut4, fcs,
	                                tm);
}

// ---------------------------------------------------------------- persistent launches
// Two persistent kernels take the tensor-core-form kinds of VDIF stations
// (plain, or raw INTERLACEDVDIF reads; of one context or of a batch of them)
// from a work list: the
// narrow one every length up to 4096 points in CTAs of 256 threads (the
// shape of k_fstage for those lengths), the wide one 8192-point FFTs of one
// band in CTAs of 512.  Each CTA takes a unit at a time from a counter and
// runs it as one CTA of k_fstage would.
constexpr size_t kNarrowSide = 36864;            // exchange buffer: 2048 points x 2 bands (or 4096 x 1), padded
constexpr size_t kWideSmem = 73728;              // 8192 points of one band, padded

template <int VAR, int NV, class Team>
__device__ __forceinline__ void narrow_unit(const FsArgs &a, const FsMultiKind &k, const FsMultiUnit &w, uint2 *fsm,
                                            const float *lut8, const float2 *lut4, FftConst *fcs, const Team &tm)
{
	const float2 *tw = (const float2 *)k.tw;
	const int gi = k.first + w.item;
	switch(k.code & 31)
	{
#define FXB_MULTI_CASE(LOGN)                                                                                   \
	case LOGN:                                                                                                 \
		fstage_unit<NV, LOGN, true, VAR>(a, gi, w.tchunk, k.tq, 0, tw, fsm, lut8, lut4, fcs, tm);             \
		break;
		FXB_MULTI_CASE(5)
		FXB_MULTI_CASE(6)
		FXB_MULTI_CASE(7)
		FXB_MULTI_CASE(8)
		FXB_MULTI_CASE(9)
		FXB_MULTI_CASE(10)
		FXB_MULTI_CASE(11)
#undef FXB_MULTI_CASE
	case 12:
		if constexpr(NV == 1)
			fstage_unit<1, 12, true, VAR>(a, gi, w.tchunk, k.tq, 0, tw, fsm, lut8, lut4, fcs, tm);
		break;
	default:
		break;
	}
}

// the next unit of this CTA (counter ctr), shared through slot
__device__ __forceinline__ int next_unit(int32_t *ctr, int *slot)
{
	if(threadIdx.x == 0)
		*slot = atomicAdd(ctr, 1);
	__syncthreads();
	const int u = *slot;
	__syncthreads();
	return u;
}

// One exchange buffer per unit (three CTAs per SM): faster than two buffers
// at two CTAs per SM on every c3 length measured.  VAR 0: plain VDIF, 1: raw
// INTERLACEDVDIF reads; NV: bands per item (an instance each keeps the
// register allocation of every length close to its own kernel's); work-list
// class 3 VAR + 3 - NV.
template <int VAR, int NV>
__global__ void __launch_bounds__(256, 3) k_fstage_pn(const __grid_constant__ FsMultiArgs m)
{
	extern __shared__ __align__(16) uint2 fsm[];
	__shared__ float lut8[256];
	__shared__ float2 lut4[16];
	__shared__ FftConst fcs[kFsMultiFc];
	__shared__ int unit_s;
	const CtaTeam cta;
	constexpr int cls = 3 * VAR + 3 - NV;
	fstage_luts(cta, true, lut8, lut4);
	for(;;)
	{
		const int u = next_unit(m.ctr + cls, &unit_s);
		if(u >= m.nunit[cls])
			break;
		const FsMultiUnit w = m.units[m.unit0[cls] + u];
		const FsMultiKind k = m.kinds[w.kind];
		narrow_unit<VAR, NV>(m.m[k.member], k, w, fsm, lut8, lut4, fcs, cta);
	}
}

// work-list class 3 VAR
template <int VAR>
__global__ void __launch_bounds__(512, 2) k_fstage_pw(const __grid_constant__ FsMultiArgs m)
{
	extern __shared__ __align__(16) uint2 fsm[];
	__shared__ float lut8[256];
	__shared__ float2 lut4[16];
	__shared__ FftConst fcs[kMaxTQ];
	__shared__ int unit_s;
	const CtaTeam cta;
	constexpr int cls = 3 * VAR;
	fstage_luts(cta, true, lut8, lut4);
	for(;;)
	{
		const int u = next_unit(m.ctr + cls, &unit_s);
		if(u >= m.nunit[cls])
			break;
		const FsMultiUnit w = m.units[m.unit0[cls] + u];
		const FsMultiKind k = m.kinds[w.kind];
		fstage_unit<1, 13, true, VAR>(m.m[k.member], k.first + w.item, w.tchunk, k.tq, 0, (const float2 *)k.tw, fsm,
		                              lut8, lut4, fcs, cta);
	}
}

bool fstage_multi_shape(int N, int nb, bool *wide)
{
	*wide = N == 8192 && nb == 1;
	return (nb == 2 && N >= 32 && N <= 2048) || (nb == 1 && N >= 32 && N <= 8192);
}

int fstage_multi_tq(int N, int nb, int tq)
{
	FKind k;
	memset(&k, 0, sizeof(k));
	if(!fstage_plan(N, nb, 1, &k))
		return 1;
	const int cap = N == 8192 ? kMaxTQ : kFsMultiFc / k.fpc;
	return tq < 1 ? 1 : (tq > cap ? cap : tq);
}

// class kernels of one read form, each on the next stream of the set
template <int VAR>
static void launch_multi_var(const FsMultiArgs &m, int nsm, const cudaStream_t *streams, int nstream, int &next)
{
	auto pick = [&]() { return streams[(next++) % nstream]; };
	// the wide units first: they are the longest
	if(m.nunit[3 * VAR] > 0)
	{
		cudaFuncSetAttribute(k_fstage_pw<VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWideSmem);
		cudaFuncSetAttribute(k_fstage_pw<VAR>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
		const int n = m.nunit[3 * VAR], grid = n < 2 * nsm ? n : 2 * nsm;
		k_fstage_pw<VAR><<<grid, 512, kWideSmem, pick()>>>(m);
	}
	auto narrow = [&](auto kern, int cls) {
		if(m.nunit[cls] <= 0)
			return;
		cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kNarrowSide);
		cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
		const int n = m.nunit[cls], grid = n < 3 * nsm ? n : 3 * nsm;
		kern<<<grid, 256, kNarrowSide, pick()>>>(m);
	};
	narrow(k_fstage_pn<VAR, 2>, 3 * VAR + 1);
	narrow(k_fstage_pn<VAR, 1>, 3 * VAR + 2);
}

cudaError_t launch_fstage_multi(const FsMultiArgs &m, int nsm, cudaStream_t stream)
{
	return launch_fstage_multi_on(m, nsm, &stream, 1);
}

cudaError_t launch_fstage_multi_on(const FsMultiArgs &m, int nsm, const cudaStream_t *streams, int nstream)
{
	int next = 0;
	launch_multi_var<0>(m, nsm, streams, nstream, next);
	launch_multi_var<1>(m, nsm, streams, nstream, next);
	return cudaGetLastError();
}

static int ilog2(int n)
{
	int l = 0;
	while((1 << l) < n)
		l++;
	return l;
}

bool fstage_plan(int N, int nb, int out, FKind *k)
{
	if(N < 32 || N > 16384 || (N & (N - 1)))
		return false;
	k->N = N;
	k->nb = nb;
	k->kb = N <= 2048 ? 1 : (N <= 8192 ? 2 : 4);
	if(nb == 2 && k->kb != 1)
		return false;                               // items of long FFTs hold one band
	const int tpf = N / (8 * k->kb);
	k->threads = tpf >= 256 ? tpf : 256;
	k->fpc = k->threads / tpf;
	const int nv = nb;
	const size_t side = (size_t)k->fpc * nv * xpad(N) * 8;
	k->pp = 2 * side <= 80 * 1024 ? 1 : 0;
	k->smem = side * (k->pp ? 2 : 1);
	k->tq = 4;
	k->out = out;
	k->items_fast = out == 1 ? 1 : 0;          // tensor-core spectra: a subband's stations side by side
	k->twn = tw_offset(N, ilog2(N) / 3);
	return k->smem <= 200 * 1024 && k->threads <= 512;
}

// Twiddle table of FFT length N in the kernel's [pass][r - 1][p] layout
// (values computed in double): n = tw_offset(N, npass) entries.
void make_fstage_twiddles(int N, float2 *out32)
{
	int n8 = N / 8, s = 1, o = 0;
	while(n8 >= 1)
	{
		for(int r = 1; r < 8; r++)
			for(int p = 0; p < n8; p++)
			{
				const double ang = -2.0 * M_PI * (double)((int64_t)r * p * s % N) / (double)N;
				out32[o + (r - 1) * n8 + p] = make_float2((float)cos(ang), (float)sin(ang));
			}
		o += 7 * n8;
		n8 /= 8;
		s *= 8;
	}
}

template <int NV, int LOGN, bool TCO, int VAR>
static void launch_t(const FKind &k, const FsArgs &a, cudaStream_t stream)
{
	cudaFuncSetAttribute(k_fstage<NV, LOGN, TCO, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
	cudaFuncSetAttribute(k_fstage<NV, LOGN, TCO, VAR>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
	const int per = k.tq * k.fpc;
	const int nt = (a.T + per - 1) / per;
	const dim3 grid = a.items_fast ? dim3(k.count, nt) : dim3(nt, k.count);
	k_fstage<NV, LOGN, TCO, VAR><<<grid, k.threads, k.smem, stream>>>(a);
}

template <int NV, bool TCO, int VAR>
static void launch_n(const FKind &k, const FsArgs &a, cudaStream_t stream)
{
	switch(k.N)
	{
	case 32: launch_t<NV, 5, TCO, VAR>(k, a, stream); break;
	case 64: launch_t<NV, 6, TCO, VAR>(k, a, stream); break;
	case 128: launch_t<NV, 7, TCO, VAR>(k, a, stream); break;
	case 256: launch_t<NV, 8, TCO, VAR>(k, a, stream); break;
	case 512: launch_t<NV, 9, TCO, VAR>(k, a, stream); break;
	case 1024: launch_t<NV, 10, TCO, VAR>(k, a, stream); break;
	case 2048: launch_t<NV, 11, TCO, VAR>(k, a, stream); break;
	default:
		if constexpr(NV == 1)
		{
			if(k.N == 4096)
				launch_t<NV, 12, TCO, VAR>(k, a, stream);
			else if(k.N == 8192)
				launch_t<NV, 13, TCO, VAR>(k, a, stream);
			else if(k.N == 16384)
				launch_t<NV, 14, TCO, VAR>(k, a, stream);
		}
		break;
	}
}

template <int VAR>
static void launch_var(const FKind &k, const FsArgs &a, cudaStream_t stream)
{
	if(k.out == 1)
	{
		if(k.nb == 2)
			launch_n<2, true, VAR>(k, a, stream);
		else
			launch_n<1, true, VAR>(k, a, stream);
	}
	else if(k.nb == 2)
		launch_n<2, false, VAR>(k, a, stream);
	else
		launch_n<1, false, VAR>(k, a, stream);
}

void launch_fstage_kind(const FKind &k, FsArgs a, cudaStream_t stream)
{
	if(k.count <= 0 || a.T <= 0)
		return;
	a.first = k.first;
	a.tq = k.tq;
	a.pp = k.pp;
	a.tw = k.tw;
	a.items_fast = k.items_fast;
	if(k.muxraw)
		launch_var<1>(k, a, stream);
	else if(k.cplx)
		launch_var<2>(k, a, stream);
	else
		launch_var<0>(k, a, stream);
}

}  // namespace fxb
