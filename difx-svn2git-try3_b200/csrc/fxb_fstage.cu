// F stage (Mode::process, mpifxcorr/src/mode.cpp:845-1308) for sm_100a.
//
// One CTA per (station, subband, chunk of TQ consecutive FFTs).  For each FFT
// of the chunk the CTA
//   1. stages the station's packed VDIF words of the FFT window in shared
//      memory (8-byte loads, frame headers skipped),
//   2. decodes the subband's one or two polarisation bands from those words
//      (2-bit / 8-bit tables of format_vdif.c:74-149), zeroing samples of
//      invalid frames and, for 8-bit 2/4-channel streams, every sample after
//      the first blanked one (format_vdif.c:1879-1922),
//   3. multiplies by the fringe rotator exp(-2 pi i phi(n)) of the order in use
//      (mode.cpp:906-1051; phi reduced to [-1/2, 1/2) turns in FP64 at the FFT
//      start, per sample in FP32),
//   4. runs a complex FFT of N = 2*nchan points as a radix-8 Stockham
//      transform in padded structure-of-arrays shared memory (one butterfly
//      per thread and pass, held in registers across the pass barrier),
//   5. selects the sideband (USB bins 0..nchan-1, LSB nchan..2nchan-1; order 0
//      takes the conjugate mirror) and applies the fractional-sample rotator
//      exp(+2 pi i f_c fse) (mode.cpp:1053-1097, 1279-1286), with the post-F
//      fringe phase for order 0 (mode.cpp:1061-1070),
//   6. writes the spectra: FP32 rows [t][row][chan] for the FP32 XMAC, or
//      BF16 K-major [chan][2*row + re/im][t] (time contiguous, the operand
//      layout of the tensor-core XMAC), staged in shared memory so that each
//      (channel, real row) receives TQ consecutive times in one store.

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

namespace {


__device__ __forceinline__ int pad(int i) { return i + (i >> 5); }

struct cf { float x, y; };

__device__ __forceinline__ cf cmulf(cf a, cf b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cf cadd(cf a, cf b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cf csub(cf a, cf b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cf mul_mi(cf a) { return {a.y, -a.x}; }   // -i * a
__device__ __forceinline__ cf mul_pi(cf a) { return {-a.y, a.x}; }   // +i * a

// forward 8-point DFT in place
__device__ __forceinline__ void dft8(cf *x)
{
	const float r = 0.70710678118654752440f;
	cf a0 = cadd(x[0], x[4]), a4 = csub(x[0], x[4]);
	cf a1 = cadd(x[1], x[5]), a5 = csub(x[1], x[5]);
	cf a2 = cadd(x[2], x[6]), a6 = csub(x[2], x[6]);
	cf a3 = cadd(x[3], x[7]), a7 = csub(x[3], x[7]);
	cf b0 = cadd(a0, a2), b2 = csub(a0, a2), b1 = cadd(a1, a3), b3 = csub(a1, a3);
	x[0] = cadd(b0, b1);
	x[4] = csub(b0, b1);
	x[2] = cadd(b2, mul_mi(b3));
	x[6] = cadd(b2, mul_pi(b3));
	cf t5 = {(a5.x + a5.y) * r, (a5.y - a5.x) * r};      // a5 * (1 - i)/sqrt2
	cf t6 = mul_mi(a6);                                  // a6 * -i
	cf t7 = {(a7.y - a7.x) * r, -(a7.x + a7.y) * r};     // a7 * (-1 - i)/sqrt2
	cf c0 = cadd(a4, t6), c2 = csub(a4, t6), c1 = cadd(t5, t7), c3 = csub(t5, t7);
	x[1] = cadd(c0, c1);
	x[5] = csub(c0, c1);
	x[3] = cadd(c2, mul_mi(c3));
	x[7] = cadd(c2, mul_pi(c3));
}

__device__ __forceinline__ void dft4(cf *x)
{
	cf b0 = cadd(x[0], x[2]), b2 = csub(x[0], x[2]), b1 = cadd(x[1], x[3]), b3 = csub(x[1], x[3]);
	x[0] = cadd(b0, b1);
	x[2] = csub(b0, b1);
	x[1] = cadd(b2, mul_mi(b3));
	x[3] = cadd(b2, mul_pi(b3));
}

__device__ __forceinline__ void dft2(cf *x)
{
	cf a = x[0], b = x[1];
	x[0] = cadd(a, b);
	x[1] = csub(a, b);
}

// One pass of the radix-R Stockham autosort FFT (decimation in frequency) on
// NB buffers at once, in place in padded SoA shared memory (buffer k: real
// part at buf + 2k padN, imaginary part at buf + (2k+1) padN);
// tw[k] = exp(-2 pi i k / maxN).  With current length len = N/s: butterfly
// (p, q), x_r = X[q + s(p + r m)], y = DFT_R(x), Y[q + s(R p + r)] =
// y_r w_len^{r p}.  Each thread holds KB butterflies per buffer in registers
// across the barrier that separates the pass's reads from its writes; the
// twiddles are shared by the buffers.
template <int R, int KB, int NB>
__device__ __forceinline__ void fft_pass(float *buf, int padN, int N, int s, int logs, const float2 *__restrict__ tw,
                                         int twscale)
{
	constexpr int logR = R == 8 ? 3 : (R == 4 ? 2 : 1);
	const int m = (N >> logs) >> logR;
	const int nb = N >> logR;
	cf y[NB][KB][R];
	int base[KB];
#pragma unroll
	for(int k = 0; k < KB; k++)
	{
		const int b = threadIdx.x + k * blockDim.x;
		base[k] = -1;
		if(b < nb)
		{
			const int q = b & (s - 1);
			const int p = b >> logs;
			cf w[R];
#pragma unroll
			for(int r = 1; r < R; r++)
			{
				const float2 t = __ldg(tw + (r * p * s) * twscale);
				w[r] = {t.x, t.y};
			}
#pragma unroll
			for(int j = 0; j < NB; j++)
			{
				const float *re = buf + 2 * j * padN, *im = re + padN;
				cf x[8];
#pragma unroll
				for(int r = 0; r < R; r++)
				{
					const int i = pad(q + s * (p + r * m));
					x[r] = {re[i], im[i]};
				}
				if(R == 8)
					dft8(x);
				else if(R == 4)
					dft4(x);
				else
					dft2(x);
				y[j][k][0] = x[0];
#pragma unroll
				for(int r = 1; r < R; r++)
					y[j][k][r] = cmulf(x[r], w[r]);
			}
			base[k] = q + s * R * p;
		}
	}
	__syncthreads();
#pragma unroll
	for(int k = 0; k < KB; k++)
		if(base[k] >= 0)
		{
#pragma unroll
			for(int j = 0; j < NB; j++)
			{
				float *re = buf + 2 * j * padN, *im = re + padN;
#pragma unroll
				for(int r = 0; r < R; r++)
				{
					const int o = pad(base[k] + s * r);
					re[o] = y[j][k][r].x;
					im[o] = y[j][k][r].y;
				}
			}
		}
	__syncthreads();
}

// Complex forward FFT of N = 2^logN points on NB buffers: radix-8 passes, then
// one radix-4 or radix-2 pass for the remaining factor.  MAXE = N / blockDim
// (>= 8) elements per buffer are held per thread in each pass.
template <int MAXE, int NB>
__device__ void fft_stockham(float *buf, int padN, int N, int logN, const float2 *__restrict__ tw, int twscale)
{
	int s = 1, logs = 0;
	while(logN - logs >= 3)
	{
		fft_pass<8, (MAXE / 8 > 0 ? MAXE / 8 : 1), NB>(buf, padN, N, s, logs, tw, twscale);
		s <<= 3;
		logs += 3;
	}
	if(logN - logs == 2)
		fft_pass<4, MAXE / 4, NB>(buf, padN, N, s, logs, tw, twscale);
	else if(logN - logs == 1)
		fft_pass<2, MAXE / 2, NB>(buf, padN, N, s, logs, tw, twscale);
}

// 2-bit code -> {-HiMag, -1, +1, +HiMag} (format_vdif.c:78) without a table:
// sign from bit 1, magnitude HiMag for codes 0 and 3
__device__ __forceinline__ float level2(uint32_t code)
{
	const float mag = ((code ^ (code >> 1)) & 1u) ? 1.0f : 3.3359f;
	return (code & 2u) ? mag : -mag;
}

__device__ __forceinline__ float frac_centered(double x)
{
	return (float)(x - rint(x));
}

}  // namespace

// Work item of the F stage: one subband (frequency) of one station, with the
// station bands recording it (at most two are processed together; a third
// band of the same frequency gets its own item).
struct FGroup {
	int32_t station, freq;
	int32_t band[2];
	int32_t row[2];          // rows within the frequency's spectra (-1: band not output)
	int32_t nb;
	int32_t lsb;
	double lofreq;
};

template <int MAXE, int OUT, int NB>
__global__ void __launch_bounds__(256, (NB == 2 && MAXE <= 8) ? 2 : 3) k_fstage2(const DevStation *__restrict__ st, const DevSubintStation *__restrict__ sub,
                                                 const FGroup *__restrict__ groups, const DevFreqPlan *__restrict__ plans,
                                                 const uint8_t *__restrict__ valid, int64_t valid_stride,
                                                 const FftParam *__restrict__ params, const float2 *__restrict__ twiddle,
                                                 int maxN, int T, int TQ, int Tpad, int order, int fractionallofreq,
                                                 int nbufmax, int rawcap_words, void *__restrict__ spec_out)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ unsigned fmask_s;
	__shared__ float lut8_s[256];

	// work item and station description, once into registers
	const FGroup *gp = groups + blockIdx.y;
	const int s = gp->station;
	const int gfreq = gp->freq;
	int band[2] = {gp->band[0], gp->band[1]};
	int row[2] = {gp->row[0], gp->row[1]};
	const bool lsb = gp->lsb != 0;
	const double lo = gp->lofreq;
	const DevStation *Sp = st + s;
	const int N = Sp->fftchannels, nchan = Sp->nchan;
	const uint32_t fs = (uint32_t)Sp->framesamples;
	const int nbits = Sp->nbits, nband = Sp->nband;
	const uint32_t payload = (uint32_t)Sp->payload;
	const int header = Sp->header, framebytes = Sp->framebytes;
	const int asl = Sp->asl;
	const double bw = Sp->bw;
	const uint8_t *buf = sub[s].buf;
	const int64_t nframes = sub[s].nbytes / framebytes;
	const int logN = 31 - __clz(N);
	const int padN = N + (N >> 5);
	float *const fbuf = (float *)smem_raw;                          // buffer k: re at 2k padN, im at (2k+1) padN
	uint32_t *raw = (uint32_t *)(fbuf + 2 * nbufmax * padN);        // staged packed words
	__nv_bfloat16 *stage = (__nv_bfloat16 *)(raw + rawcap_words);   // OUT == 1: [NB*2][TQ][nchan]
	const uint8_t *vrow = valid + (int64_t)s * valid_stride;
	const int twscale = maxN / N;
	const uint32_t bits_per_time = (uint32_t)(nband * nbits);
	const int64_t spec_off = plans[gfreq].spec_off;
	const int prow = plans[gfreq].nrow;
	const int r2pad = plans[gfreq].r2pad;
	const int t0 = blockIdx.x * TQ;
	const int tq_n = min(TQ, T - t0);
	if(nbits == 8)
	{
		// (b - 128) / 3.3 in double, rounded to float (format_vdif.c:122)
		for(int i = threadIdx.x; i < 256; i += blockDim.x)
			lut8_s[i] = (float)((i - 128) / 3.3);
	}

	for(int tq = 0; tq < tq_n; tq++)
	{
		const int t = t0 + tq;
		const FftParam p = params[(int64_t)s * T + t];
		if(p.status != kFftOk)
		{
#pragma unroll
			for(int k = 0; k < NB; k++)
				for(int c = threadIdx.x; c < nchan; c += blockDim.x)
				{
					if(OUT == 0)
					{
						if(row[k] >= 0)
							((float2 *)spec_out)[spec_off + ((int64_t)t * prow + row[k]) * nchan + c] =
							    make_float2(0.0f, 0.0f);
					}
					else
					{
						stage[((size_t)(2 * k) * TQ + tq) * nchan + c] = __float2bfloat16_rn(0.0f);
						stage[((size_t)(2 * k + 1) * TQ + tq) * nchan + c] = __float2bfloat16_rn(0.0f);
					}
				}
			continue;
		}
		// ---- 1. stage the packed words of the window [nearest, nearest + N)
		// (all offsets fit in 32 bits: a station buffer holds < 2^31 samples)
		const uint32_t g0 = (uint32_t)p.nearest;
		const uint32_t fa = g0 / fs;
		const uint32_t so = g0 - fa * fs;                               // window start in stream samples
		const uint32_t sb0 = ((so * bits_per_time) >> 3) & ~7u;         // first staged byte (8-aligned)
		const uint32_t sbe = ((so + (uint32_t)N) * bits_per_time + 7) >> 3;
		const int nw8 = (int)((sbe - sb0 + 7) >> 3);
		const bool staged = 2 * nw8 <= rawcap_words;
		const int nwf = (int)((so + (uint32_t)N - 1) / fs) + 1;           // frames touched by the window
		if(staged)
		{
			uint32_t sb = sb0 + 8u * threadIdx.x;
			uint32_t k = sb / payload;
			uint32_t off = sb - k * payload;
			for(int w = threadIdx.x; w < nw8; w += blockDim.x)
			{
				const int64_t fr = (int64_t)fa + k;
				uint2 v = make_uint2(0u, 0u);
				if(fr < nframes)
					v = __ldg((const uint2 *)(buf + fr * framebytes + header + off));
				raw[2 * w] = v.x;
				raw[2 * w + 1] = v.y;
				off += 8u * blockDim.x;
				while(off >= payload)
				{
					off -= payload;
					k++;
				}
			}
		}
		if(threadIdx.x < 32)
		{
			// validity of the window's frames, one bit per frame (nwf <= 32)
			const int64_t fr = (int64_t)fa + threadIdx.x;
			const bool v = threadIdx.x < nwf && fr < valid_stride && vrow[fr];
			const unsigned m = __ballot_sync(0xffffffffu, v);
			if(threadIdx.x == 0)
				fmask_s = m;
		}
		__syncthreads();
		// ---- 2/3. decode, rotate into the FFT buffers
		const double fraclo = fractionallofreq ? (lo - (int)lo) * (double)p.integerdelay : 0.0;
		float P0 = 0.0f, alpha = 0.0f, beta = 0.0f, gamma = 0.0f, eps = 0.0f;
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
		const uint32_t fmask = fmask_s;
		const bool wide = nwf > 32;                                       // tiny frames: look validity up per sample
		const uint32_t bitbase = so * bits_per_time - sb0 * 8u;
		const int stuck = p.stuck;
		uint32_t boff[NB];
#pragma unroll
		for(int k = 0; k < NB; k++)
			boff[k] = (uint32_t)(band[k] * nbits);
		uint32_t kf = (so + threadIdx.x) / fs;                           // frame of the thread's sample (rel. fa)
		uint32_t kend = (kf + 1) * fs - so;                               // window index where that frame ends
		for(int n = threadIdx.x; n < N; n += blockDim.x)
		{
			while((uint32_t)n >= kend)
			{
				kf++;
				kend += fs;
			}
			bool ok = wide ? ((int64_t)fa + kf < valid_stride && vrow[(int64_t)fa + kf]) : ((fmask >> kf) & 1u);
			ok = ok && n < stuck;
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
			const uint32_t nbit = bitbase + (uint32_t)n * bits_per_time;
#pragma unroll
			for(int k = 0; k < NB; k++)
			{
				float v = 0.0f;
				if(ok)
				{
					if(staged)
					{
						const uint32_t bit = nbit + boff[k];
						const uint32_t word = raw[bit >> 5] >> (bit & 31);
						v = nbits == 2 ? level2(word & 3u) : lut8_s[word & 255u];
					}
					else
					{
						const int64_t fr = (int64_t)fa + kf;
						const int64_t tin = (int64_t)so + n - (int64_t)kf * fs;
						const uint8_t *plb = buf + fr * framebytes + header;
						const int64_t q = tin * nband + band[k];
						if(nbits == 2)
						{
							const int64_t bit = q * 2;
							v = level2((__ldg(plb + (bit >> 3)) >> (bit & 7)) & 3u);
						}
						else
							v = lut8_s[__ldg(plb + q)];
					}
				}
				fbuf[2 * k * padN + pad(n)] = v * cs;
				fbuf[(2 * k + 1) * padN + pad(n)] = v * sn;
			}
		}
		__syncthreads();
		// ---- 4. FFTs of the NB bands together
		fft_stockham<MAXE, NB>(fbuf, padN, N, logN, twiddle, twscale);
		// ---- 5/6. sideband, fractional-sample rotation, output
		const float dfs = (float)(bw / nchan * (double)p.fse);
		float postf = 0.0f;
		if(order == 0)
		{
			double pr = (p.averagedelay - p.integerdelay) * lo;
			if(fractionallofreq)
				pr += p.integerdelay * (lo - (int)lo);
			postf = -(float)(pr - (int)pr);
		}
		for(int c = threadIdx.x; c < nchan; c += blockDim.x)
		{
			int src, ce;
			float conj = 1.0f;
			if(lsb)
			{
				ce = c - nchan;
				if(order == 0)
				{
					src = nchan - c;
					conj = -1.0f;
				}
				else
					src = nchan + c;
			}
			else
			{
				ce = c;
				src = c;
			}
			float turns = (float)ce * dfs + postf;
			turns -= rintf(turns);
			float sn, cs;
			__sincosf(6.283185307179586f * turns, &sn, &cs);
			const int ps = pad(src);
#pragma unroll
			for(int k = 0; k < NB; k++)
			{
				const float xr = fbuf[2 * k * padN + ps], xi = conj * fbuf[(2 * k + 1) * padN + ps];
				const float yr = xr * cs - xi * sn, yi = xr * sn + xi * cs;
				if(OUT == 0)
				{
					if(row[k] >= 0)
						((float2 *)spec_out)[spec_off + ((int64_t)t * prow + row[k]) * nchan + c] = make_float2(yr, yi);
				}
				else
				{
					stage[((size_t)(2 * k) * TQ + tq) * nchan + c] = __float2bfloat16_rn(yr);
					stage[((size_t)(2 * k + 1) * TQ + tq) * nchan + c] = __float2bfloat16_rn(yi);
				}
			}
		}
		__syncthreads();
	}
	if(OUT == 1)
	{
		// [chan][2 row + part][Tpad] bf16: each (channel, real row) receives the
		// chunk's TQ consecutive times in one 16-byte store
		__nv_bfloat16 *o = (__nv_bfloat16 *)spec_out;
		const int nitems = NB * 2 * nchan;
		for(int it = threadIdx.x; it < nitems; it += blockDim.x)
		{
			const int c = it % nchan;
			const int kp = it / nchan;            // k * 2 + part
			const int k = kp >> 1, part = kp & 1;
			const int rk = k == 0 ? row[0] : row[1];
			if(rk < 0)
				continue;
			__nv_bfloat16 *dst = o + spec_off + ((int64_t)c * r2pad + 2 * rk + part) * Tpad + t0;
			const __nv_bfloat16 *src = stage + (size_t)kp * TQ * nchan + c;
			if(TQ == 8 && tq_n == 8)
			{
				__align__(16) __nv_bfloat16 v[8];
#pragma unroll
				for(int q = 0; q < 8; q++)
					v[q] = src[(size_t)q * nchan];
				*(uint4 *)dst = *(const uint4 *)v;
			}
			else
				for(int q = 0; q < tq_n; q++)
					dst[q] = src[(size_t)q * nchan];
		}
	}
}

size_t fstage2_smem(int N, int nband, int nbits, int nchan, int out, int TQ, int nbufmax, int *rawcap_words)
{
	const int padN = N + (N >> 5);
	size_t fft = (size_t)2 * nbufmax * padN * sizeof(float);
	// raw window: N samples x bits + 16 bytes slack, capped at 48 KB
	size_t rawb = ((size_t)N * nband * nbits + 7) / 8 + 32;
	if(rawb > 48 * 1024)
		rawb = 0;                    // decode from global memory instead
	rawb = (rawb + 15) & ~(size_t)15;
	*rawcap_words = (int)(rawb / 4);
	size_t stg = out == 1 ? (size_t)2 * 2 * nchan * TQ * sizeof(__nv_bfloat16) : 0;
	return fft + rawb + stg;
}

template <int MAXE, int OUT, int NB>
static void launch_one(dim3 grid, size_t smem, cudaStream_t stream, const DevStation *st, const DevSubintStation *sub,
                       const FGroup *groups, const DevFreqPlan *plans, const uint8_t *valid, int64_t valid_stride,
                       const FftParam *params, const float2 *twiddle, int maxN, int T, int TQ, int Tpad, int order,
                       int fraclo, int nbufmax, int rawcap, void *out)
{
	cudaFuncSetAttribute(k_fstage2<MAXE, OUT, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
	k_fstage2<MAXE, OUT, NB><<<grid, 256, smem, stream>>>(st, sub, groups, plans, valid, valid_stride, params, twiddle,
	                                                        maxN, T, TQ, Tpad, order, fraclo, nbufmax, rawcap, out);
}

template <int MAXE>
static void launch_maxe(int npair, int nsingle, int Tchunks, size_t smem, cudaStream_t stream, const DevStation *st,
                        const DevSubintStation *sub, const FGroup *g, const DevFreqPlan *plans, const uint8_t *valid,
                        int64_t valid_stride, const FftParam *params, const float2 *twiddle, int maxN, int T, int TQ,
                        int Tpad, int order, int fl, int nbufmax, int rawcap, int out, void *spec)
{
	if(npair > 0)
	{
		dim3 grid(Tchunks, npair);
		if(out == 0)
			launch_one<MAXE, 0, 2>(grid, smem, stream, st, sub, g, plans, valid, valid_stride, params, twiddle, maxN, T,
			                       TQ, Tpad, order, fl, nbufmax, rawcap, spec);
		else
			launch_one<MAXE, 1, 2>(grid, smem, stream, st, sub, g, plans, valid, valid_stride, params, twiddle, maxN, T,
			                       TQ, Tpad, order, fl, nbufmax, rawcap, spec);
	}
	if(nsingle > 0)
	{
		dim3 grid(Tchunks, nsingle);
		if(out == 0)
			launch_one<MAXE, 0, 1>(grid, smem, stream, st, sub, g + npair, plans, valid, valid_stride, params, twiddle,
			                       maxN, T, TQ, Tpad, order, fl, nbufmax, rawcap, spec);
		else
			launch_one<MAXE, 1, 1>(grid, smem, stream, st, sub, g + npair, plans, valid, valid_stride, params, twiddle,
			                       maxN, T, TQ, Tpad, order, fl, nbufmax, rawcap, spec);
	}
}

void launch_fstage2(const DevStation *st, const DevSubintStation *sub, const void *groups, int npair, int nsingle,
                    const DevFreqPlan *plans, const uint8_t *valid, int64_t valid_stride, const FftParam *params,
                    const float2 *twiddle, int maxN, int T, int TQ, int Tpad, int order, bool fractionallofreq,
                    int N, int nband_max, int nbits_max, int nbufmax, int out, void *spec, cudaStream_t stream)
{
	int rawcap = 0;
	size_t smem = fstage2_smem(N, nband_max, nbits_max, N / 2, out, TQ, nbufmax, &rawcap);
	const int me = N / 256;     // elements per thread and pass
	const FGroup *g = (const FGroup *)groups;
	const int fl = fractionallofreq ? 1 : 0;
	const int tch = (T + TQ - 1) / TQ;
	if(me <= 8)
		launch_maxe<8>(npair, nsingle, tch, smem, stream, st, sub, g, plans, valid, valid_stride, params, twiddle, maxN,
		               T, TQ, Tpad, order, fl, nbufmax, rawcap, out, spec);
	else if(me <= 16)
		launch_maxe<16>(npair, nsingle, tch, smem, stream, st, sub, g, plans, valid, valid_stride, params, twiddle, maxN,
		                T, TQ, Tpad, order, fl, nbufmax, rawcap, out, spec);
	else if(me <= 32)
		launch_maxe<32>(npair, nsingle, tch, smem, stream, st, sub, g, plans, valid, valid_stride, params, twiddle, maxN,
		                T, TQ, Tpad, order, fl, nbufmax, rawcap, out, spec);
	else
		launch_maxe<64>(npair, nsingle, tch, smem, stream, st, sub, g, plans, valid, valid_stride, params, twiddle, maxN,
		                T, TQ, Tpad, order, fl, nbufmax, rawcap, out, spec);
}

size_t fgroup_size() { return sizeof(FGroup); }

void make_fgroup(void *dst, int station, int freq, int b0, int b1, int r0, int r1, int lsb, double lofreq)
{
	FGroup g;
	g.station = station;
	g.freq = freq;
	g.band[0] = b0;
	g.band[1] = b1 < 0 ? b0 : b1;
	g.row[0] = r0;
	g.row[1] = r1;
	g.nb = b1 < 0 ? 1 : 2;
	g.lsb = lsb;
	g.lofreq = lofreq;
	*(FGroup *)dst = g;
}

}  // namespace fxb
