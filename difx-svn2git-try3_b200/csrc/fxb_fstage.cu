// F stage (Mode::process, mpifxcorr/src/mode.cpp:845-1308) for sm_100a.
//
// One CTA per (station, subband, chunk of FFTs); a subband's one or two
// polarisation bands are transformed together.  Each thread owns KB radix-8
// butterflies of every pass of one FFT ("slot"): an FFT of N points takes
// N / (8 KB) threads, and a CTA runs several slots side by side when N is
// small.  Per FFT a thread
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
// Two arithmetic forms:
//   out 0: FP32 FFT, spectra as float2 (the plain FP32 form);
//   out 1: FP16 FFT with the two bands packed in half2 lanes (one instruction
//          advances both polarisations), spectra as bf16x2 (re, im) for the
//          tensor-core XMAC.  Samples are scaled by 2^-e so that no FFT value
//          can leave the FP16 range; the outputs are scaled back exactly.

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
__host__ __device__ __forceinline__ int xpad(int i) { return i + 2 * (i >> 4); }

// ---- lane values: FP32 complex (one band), packed FP16 complex (two bands)
struct cf { float x, y; };
struct hc { __half2 x, y; };      // x = (re band0, re band1), y = (im band0, im band1)
struct hw { __half2 r, i; };      // twiddle as (wr, wr), (wi, wi)

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

__device__ __forceinline__ hc add(hc a, hc b) { return {__hadd2(a.x, b.x), __hadd2(a.y, b.y)}; }
__device__ __forceinline__ hc sub(hc a, hc b) { return {__hsub2(a.x, b.x), __hsub2(a.y, b.y)}; }
__device__ __forceinline__ hc add_mi(hc a, hc b) { return {__hadd2(a.x, b.y), __hsub2(a.y, b.x)}; }
__device__ __forceinline__ hc add_pi(hc a, hc b) { return {__hsub2(a.x, b.y), __hadd2(a.y, b.x)}; }
__device__ __forceinline__ hc rot45(hc a)
{
	const __half2 r = __float2half2_rn(0.70710678118654752440f);
	return {__hmul2(__hadd2(a.x, a.y), r), __hmul2(__hsub2(a.y, a.x), r)};
}
__device__ __forceinline__ hc twid(hc a, hw w)
{
	return {__hfma2(a.x, w.r, __hneg2(__hmul2(a.y, w.i))), __hfma2(a.x, w.i, __hmul2(a.y, w.r))};
}

__device__ __forceinline__ float2 ldtw(const float2 *t, int i) { return __ldg(t + i); }
__device__ __forceinline__ hw ldtw(const hw *t, int i)
{
	const uint2 u = __ldg((const uint2 *)t + i);
	hw w;
	w.r = *(const __half2 *)&u.x;
	w.i = *(const __half2 *)&u.y;
	return w;
}

// 8-byte shared-memory element <-> lane value
template <typename C> __device__ __forceinline__ C lds(const uint2 *p);
template <> __device__ __forceinline__ cf lds<cf>(const uint2 *p)
{
	const float2 v = *(const float2 *)p;
	return {v.x, v.y};
}
template <> __device__ __forceinline__ hc lds<hc>(const uint2 *p)
{
	const uint2 u = *p;
	hc v;
	v.x = *(const __half2 *)&u.x;
	v.y = *(const __half2 *)&u.y;
	return v;
}
__device__ __forceinline__ uint2 bits(cf v) { return make_uint2(__float_as_uint(v.x), __float_as_uint(v.y)); }
__device__ __forceinline__ uint2 bits(hc v) { return make_uint2(*(const uint32_t *)&v.x, *(const uint32_t *)&v.y); }
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
	if(R == 8)
		dft8(x);
	else if(R == 4)
		dft4(x);
	else
		dft2(x);
}

// 2-bit code -> {-HiMag, -1, +1, +HiMag} (format_vdif.c:78): sign from bit 1,
// magnitude HiMag for codes 0 and 3
__device__ __forceinline__ float level2(uint32_t code)
{
	const float mag = ((code ^ (code >> 1)) & 1u) ? 1.0f : 3.3359f;
	return (code & 2u) ? mag : -mag;
}

__device__ __forceinline__ float frac_centered(double x) { return (float)(x - rint(x)); }

// per-FFT constants of one slot
struct SlotConst {
	int t;
	bool tok;         // t < T
	float dfs;        // fractional-sample rotation turns per channel
	float postf;      // order-0 post-F fringe turns
};

// One radix-8 butterfly of a middle pass (stride s = 2^logs, m = N / (8 s)):
// x_r = X[q + s (p + r m)], y = DFT8(x), y_r *= w_N^(r p s).
template <typename C, int NV, typename TW>
__device__ __forceinline__ void radix8_step(const uint2 *src, int padN, int q, int s, int p8, int m, const TW *tw,
                                            int twscale, C (&x)[NV][8])
{
#pragma unroll
	for(int j = 0; j < NV; j++)
	{
#pragma unroll
		for(int r = 0; r < 8; r++)
			x[j][r] = lds<C>(src + j * padN + xpad(q + s * (p8 + r * m)));
		dft8(x[j]);
	}
#pragma unroll
	for(int r = 1; r < 8; r++)
	{
		const TW w = ldtw(tw, r * p8 * s * twscale);
#pragma unroll
		for(int j = 0; j < NV; j++)
			x[j][r] = twid(x[j][r], w);
	}
}

// Output of the last pass (radix R, stride sL = N/R, no twiddles): bins
// q + sL r of the butterflies q = bt + j TPF go to their channels.
template <typename C, int NV, int KB, int R>
__device__ __forceinline__ void last_pass(const uint2 *src, int padN, int N, int nchan, int TPF, int bt, bool lsb,
                                          int order, const SlotConst &sc, const int row[2], int prow,
                                          int64_t spec_off, float hout, void *spec)
{
	constexpr bool H = std::is_same<C, hc>::value;
	constexpr int J = (KB * 8) / R;
	const int sL = N / R;
#pragma unroll
	for(int jj = 0; jj < J; jj++)
	{
		const int q = bt + jj * TPF;
		C y[NV][R];
#pragma unroll
		for(int j = 0; j < NV; j++)
		{
#pragma unroll
			for(int r = 0; r < R; r++)
				y[j][r] = lds<C>(src + j * padN + xpad(q + sL * r));
			dftR<R>(y[j]);
		}
#pragma unroll
		for(int r = 0; r < R; r++)
		{
			const int k = q + sL * r;
			int c, ce;
			bool use;
			float cj = 1.0f;
			if(!lsb)
			{
				use = k < nchan;
				c = k;
				ce = k;
			}
			else if(order != 0)
			{
				use = k >= nchan;
				c = k - nchan;
				ce = c - nchan;
			}
			else
			{
				use = k >= 1 && k <= nchan;
				c = nchan - k;
				ce = c - nchan;
				cj = -1.0f;
			}
			if(!use || !sc.tok)
				continue;
			float turns = (float)ce * sc.dfs + sc.postf;
			turns -= rintf(turns);
			float sn, cs;
			__sincosf(6.283185307179586f * turns, &sn, &cs);
			const int64_t o0 = spec_off + ((int64_t)sc.t * prow) * nchan + c;
			if constexpr(H)
			{
				const hc v = y[0][r];
				const float xr[2] = {__low2float(v.x) * hout, __high2float(v.x) * hout};
				const float xi[2] = {cj * __low2float(v.y) * hout, cj * __high2float(v.y) * hout};
#pragma unroll
				for(int b = 0; b < 2; b++)
					if(row[b] >= 0)
						((__nv_bfloat162 *)spec)[o0 + (int64_t)row[b] * nchan] =
						    __floats2bfloat162_rn(xr[b] * cs - xi[b] * sn, xr[b] * sn + xi[b] * cs);
			}
			else
			{
#pragma unroll
				for(int j = 0; j < NV; j++)
					if(row[j] >= 0)
					{
						const cf v = y[j][r];
						const float xr = v.x, xi = cj * v.y;
						((float2 *)spec)[o0 + (int64_t)row[j] * nchan] = make_float2(xr * cs - xi * sn, xr * sn + xi * cs);
					}
			}
		}
	}
}

}  // namespace

// C: lane type (cf: FP32, one band per value; hc: FP16, both bands per value)
// NV: values per point (cf: bands of the item; hc: 1); KB: butterflies per
// thread and radix-8 pass.
template <typename C, int NV, int KB>
__global__ void __launch_bounds__(KB == 4 ? 512 : 256, KB == 4 ? 1 : 2) k_fstage(const FsArgs a)
{
	using TW = typename std::conditional<std::is_same<C, hc>::value, hw, float2>::type;
	constexpr bool H = std::is_same<C, hc>::value;
	extern __shared__ __align__(16) uint2 fsm[];
	__shared__ float lut8[256];

	const FGroup g = a.groups[a.first + blockIdx.y];
	const DevStation *Sp = a.st + g.station;
	const int N = Sp->fftchannels, nchan = Sp->nchan;
	const uint32_t fs = (uint32_t)Sp->framesamples;
	const int nbits = Sp->nbits;
	const uint32_t bpt = (uint32_t)(Sp->nband * nbits);
	const int header = Sp->header, framebytes = Sp->framebytes, asl = Sp->asl;
	const double bw = Sp->bw;
	const uint8_t *buf = a.sub[g.station].buf;
	const int64_t nframes = a.sub[g.station].nbytes / framebytes;
	const int logN = 31 - __clz(N);
	const int padN = xpad(N);
	const int TPF = N / (8 * KB);
	const int FPC = blockDim.x / TPF;
	const int slot = threadIdx.x / TPF, bt = threadIdx.x - slot * TPF;
	uint2 *const side0 = fsm + (size_t)slot * NV * padN;
	uint2 *const side1 = a.pp ? side0 + (size_t)FPC * NV * padN : side0;
	const uint8_t *vrow = a.valid + (int64_t)g.station * a.valid_stride;
	const int twscale = a.maxN / N;
	const TW *tw = (const TW *)a.tw;
	const int64_t spec_off = a.plans[g.freq].spec_off;
	const int prow = a.plans[g.freq].nrow;
	const bool lsb = g.lsb != 0;
	const double lo = g.lofreq;
	const int row[2] = {g.row[0], g.row[1]};
	const uint32_t boff0 = (uint32_t)(g.band[0] * nbits), boff1 = (uint32_t)(g.band[1] * nbits);
	const bool oneword = bpt <= 32;       // all bands of a sample time in one 32-bit word
	const int order = a.order;
	int hexp = 0;
	if(H)
	{
		// largest |X| is N times the largest level; keep it below 2^15
		const float lvl = nbits == 2 ? 3.3359f : 38.8f;
		while(lvl * (float)N > 32768.0f * (float)(1 << hexp))
			hexp++;
	}
	const float hin = H ? ldexpf(1.0f, -hexp) : 1.0f, hout = H ? ldexpf(1.0f, hexp) : 1.0f;
	if(nbits == 8)
	{
		// (b - 128) / 3.3 in double, rounded to float (format_vdif.c:122)
		for(int i = threadIdx.x; i < 256; i += blockDim.x)
			lut8[i] = (float)((i - 128) / 3.3);
	}
	__syncthreads();

	const int t0 = blockIdx.x * a.tq * FPC;
	const int nit = min(a.tq, (a.T - t0 + FPC - 1) / FPC);
	int wb = 0;
	for(int it = 0; it < nit; it++)
	{
		SlotConst sc;
		sc.t = t0 + it * FPC + slot;
		sc.tok = sc.t < a.T;
		FftParam p;
		if(sc.tok)
			p = a.params[(int64_t)g.station * a.T + sc.t];
		const bool active = sc.tok && p.status == kFftOk;
		// ---- 1/2. decode and fringe-rotate x[b + r N/8] into registers
		uint32_t fa = 0, so = 0;
		int stuck = 0;
		float P0 = 0.0f, alpha = 0.0f, beta = 0.0f, gamma = 0.0f, eps = 0.0f;
		sc.dfs = 0.0f;
		sc.postf = 0.0f;
		if(active)
		{
			const uint32_t g0 = (uint32_t)p.nearest;
			fa = g0 / fs;
			so = g0 - fa * fs;
			stuck = p.stuck;
			const double fraclo = a.fraclo ? (lo - (int)lo) * (double)p.integerdelay : 0.0;
			if(order == 1)
			{
				P0 = frac_centered(lo * p.b + fraclo);
				alpha = (float)(lo * p.a / N);
			}
			else if(order == 2)
			{
				const double X1 = (double)asl / (double)N;
				P0 = frac_centered(lo * p.c + fraclo);
				alpha = (float)(lo * (p.b + p.a * X1) / N);
				beta = (float)(lo * 2.0 * p.a * X1 / N);
				gamma = (float)(lo * p.b * asl / N);
				eps = (float)(lo * p.a * X1 * X1);
			}
			sc.dfs = (float)(bw / nchan * (double)p.fse);
			if(order == 0)
			{
				double pr = (p.averagedelay - p.integerdelay) * lo;
				if(a.fraclo)
					pr += p.integerdelay * (lo - (int)lo);
				sc.postf = -(float)(pr - (int)pr);
			}
		}
		// ---- 1-3. decode, fringe-rotate and run the first radix-8 pass (s = 1:
		// butterfly b, twiddle w_N^(r b)), one butterfly at a time
		{
			uint2 *dst = wb ? side1 : side0;
			if(!a.pp)
				__syncthreads();              // the single buffer has been read by the last FFT
#pragma unroll
			for(int k = 0; k < KB; k++)
			{
				const int b = bt + k * TPF;
				const uint32_t xs = so + (uint32_t)b;
				uint32_t kf = xs / fs, tin = xs - kf * fs;
				C x[NV][8];
#pragma unroll
				for(int r = 0; r < 8; r++)
				{
					const int n = b + r * (N >> 3);
					const int64_t fr = (int64_t)fa + kf;
					bool ok = active && n < stuck && fr < nframes && fr < a.valid_stride;
					ok = ok && __ldg(vrow + fr) != 0;
					float v0 = 0.0f, v1 = 0.0f;
					if(ok)
					{
						const uint32_t *wp = (const uint32_t *)(buf + fr * framebytes + header);
						const uint32_t bit0 = tin * bpt + boff0;
						const uint32_t raw0 = __ldg(wp + (bit0 >> 5));
						const uint32_t w0 = raw0 >> (bit0 & 31u);
						v0 = nbits == 2 ? level2(w0 & 3u) : lut8[w0 & 255u];
						if(H || NV == 2)
						{
							const uint32_t bit1 = tin * bpt + boff1;
							const uint32_t w1 = (oneword ? raw0 : __ldg(wp + (bit1 >> 5))) >> (bit1 & 31u);
							v1 = nbits == 2 ? level2(w1 & 3u) : lut8[w1 & 255u];
						}
					}
					float sn = 0.0f, cs = 1.0f;
					if(order != 0)
					{
						float ph;
						if(order == 1)
							ph = P0 + (float)n * alpha;
						else
						{
							const int kk = n / asl, jj = n - kk * asl;
							ph = P0 + (float)jj * alpha + (float)(kk * jj) * beta + (float)kk * gamma + (float)(kk * kk) * eps;
						}
						ph -= rintf(ph);
						__sincosf(-6.283185307179586f * ph, &sn, &cs);
					}
					if constexpr(H)
					{
						x[0][r].x = __floats2half2_rn(v0 * cs * hin, v1 * cs * hin);
						x[0][r].y = __floats2half2_rn(v0 * sn * hin, v1 * sn * hin);
					}
					else
					{
						x[0][r] = cf{v0 * cs, v0 * sn};
						if constexpr(NV == 2)
							x[1][r] = cf{v1 * cs, v1 * sn};
					}
					tin += (uint32_t)(N >> 3);
					while(tin >= fs)
					{
						tin -= fs;
						kf++;
					}
				}
#pragma unroll
				for(int j = 0; j < NV; j++)
					dft8(x[j]);
#pragma unroll
				for(int r = 1; r < 8; r++)
				{
					const TW w = ldtw(tw, r * b * twscale);
#pragma unroll
					for(int j = 0; j < NV; j++)
						x[j][r] = twid(x[j][r], w);
				}
				const int o = xpad(8 * b);
#pragma unroll
				for(int j = 0; j < NV; j++)
				{
					uint2 *q = dst + j * padN + o;
					sts2(q, x[j][0], x[j][1]);
					sts2(q + 2, x[j][2], x[j][3]);
					sts2(q + 4, x[j][4], x[j][5]);
					sts2(q + 6, x[j][6], x[j][7]);
				}
			}
			__syncthreads();
		}
		// ---- middle radix-8 passes through shared memory
		int logs = 3;
		const int nmid = (logN % 3 == 0) ? logN / 3 - 2 : logN / 3 - 1;
		for(int ps = 0; ps < nmid; ps++)
		{
			const int s = 1 << logs;
			const int m = N >> (logs + 3);
			const uint2 *src = wb ? side1 : side0;
			wb ^= 1;
			uint2 *dst = wb ? side1 : side0;
			if(a.pp)
			{
				// two buffers: each butterfly reads, transforms and writes on its own
#pragma unroll
				for(int k = 0; k < KB; k++)
				{
					const int b = bt + k * TPF;
					const int q = b & (s - 1), p8 = b >> logs;
					C x[NV][8];
					radix8_step<C, NV>(src, padN, q, s, p8, m, tw, twscale, x);
#pragma unroll
					for(int j = 0; j < NV; j++)
#pragma unroll
						for(int r = 0; r < 8; r++)
							sts(dst + j * padN + xpad(q + s * (8 * p8 + r)), x[j][r]);
				}
			}
			else
			{
				// one buffer: all reads of the pass before any write
				C x[KB][NV][8];
#pragma unroll
				for(int k = 0; k < KB; k++)
				{
					const int b = bt + k * TPF;
					radix8_step<C, NV>(src, padN, b & (s - 1), s, b >> logs, m, tw, twscale, x[k]);
				}
				__syncthreads();
#pragma unroll
				for(int k = 0; k < KB; k++)
				{
					const int b = bt + k * TPF;
					const int q = b & (s - 1), p8 = b >> logs;
#pragma unroll
					for(int j = 0; j < NV; j++)
#pragma unroll
						for(int r = 0; r < 8; r++)
							sts(dst + j * padN + xpad(q + s * (8 * p8 + r)), x[k][j][r]);
				}
			}
			__syncthreads();
			logs += 3;
		}
		// ---- 4. last pass, sideband selection, fractional-sample rotation, output
		{
			const uint2 *src = wb ? side1 : side0;
			const int rl = logN - logs;
			if(rl == 3)
				last_pass<C, NV, KB, 8>(src, padN, N, nchan, TPF, bt, lsb, order, sc, row, prow, spec_off, hout, a.spec);
			else if(rl == 2)
				last_pass<C, NV, KB, 4>(src, padN, N, nchan, TPF, bt, lsb, order, sc, row, prow, spec_off, hout, a.spec);
			else
				last_pass<C, NV, KB, 2>(src, padN, N, nchan, TPF, bt, lsb, order, sc, row, prow, spec_off, hout, a.spec);
			wb ^= 1;
		}
	}
}

bool fstage_plan(int N, int nb, int out, FKind *k)
{
	k->N = N;
	k->nb = nb;
	k->kb = N <= 2048 ? 1 : (N == 4096 ? 2 : 4);
	if(out == 0 && nb == 2 && k->kb != 1)
		return false;                               // FP32 items of long FFTs hold one band
	const int tpf = N / (8 * k->kb);
	k->threads = tpf >= 256 ? tpf : 256;
	k->fpc = k->threads / tpf;
	const int nv = out == 1 ? 1 : nb;
	const size_t side = (size_t)k->fpc * nv * xpad(N) * 8;
	k->pp = 2 * side <= 80 * 1024 ? 1 : 0;
	k->smem = side * (k->pp ? 2 : 1);
	k->tq = 4;
	k->out = out;
	return k->smem <= 200 * 1024 && k->threads <= 512;
}

template <typename C, int NV, int KB>
static void launch_t(const FKind &k, int T, const FsArgs &a, cudaStream_t stream)
{
	cudaFuncSetAttribute(k_fstage<C, NV, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
	const int per = k.tq * k.fpc;
	dim3 grid((T + per - 1) / per, k.count);
	k_fstage<C, NV, KB><<<grid, k.threads, k.smem, stream>>>(a);
}

void launch_fstage_kind(const FKind &k, FsArgs a, cudaStream_t stream)
{
	if(k.count <= 0 || a.T <= 0)
		return;
	a.first = k.first;
	a.tq = k.tq;
	a.pp = k.pp;
	if(k.out == 1)
	{
		if(k.kb == 1)
			launch_t<hc, 1, 1>(k, a.T, a, stream);
		else if(k.kb == 2)
			launch_t<hc, 1, 2>(k, a.T, a, stream);
		else
			launch_t<hc, 1, 4>(k, a.T, a, stream);
	}
	else if(k.nb == 2)
		launch_t<cf, 2, 1>(k, a.T, a, stream);
	else if(k.kb == 1)
		launch_t<cf, 1, 1>(k, a.T, a, stream);
	else if(k.kb == 2)
		launch_t<cf, 1, 2>(k, a.T, a, stream);
	else
		launch_t<cf, 1, 4>(k, a.T, a, stream);
}

void make_fstage_twiddles16(const double *re, const double *im, int n, void *out)
{
	uint2 *o = (uint2 *)out;
	for(int i = 0; i < n; i++)
	{
		const __half r = __double2half(re[i]), q = __double2half(im[i]);
		const __half2 rr = __halves2half2(r, r), qq = __halves2half2(q, q);
		o[i].x = *(const uint32_t *)&rr;
		o[i].y = *(const uint32_t *)&qq;
	}
}

}  // namespace fxb
