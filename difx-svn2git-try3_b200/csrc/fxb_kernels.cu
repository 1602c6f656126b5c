// sm_100a kernels of the FX path: fused F stage, FP32 XMAC, weights,
// finalisation into the core-result layout, and the stand-alone VDIF decoder.

#include <cuda_runtime.h>
#include <cstdint>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

// 2-bit code -> level, {-HiMag, -1, +1, +HiMag} with HiMag = 3.3359
// (libraries/mark5access/mark5access/format_vdif.c:48,78; mark5_stream.h:75).
__constant__ float c_lut2[4] = {-3.3359f, -1.0f, 1.0f, 3.3359f};
// 8-bit offset binary -> (b - 128) / 3.3 (format_vdif.c:122), filled from the host.
__constant__ float c_lut8[256];

cudaError_t upload_lut8(cudaStream_t stream);

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
	return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Sample (station-relative index g) of band `band`; 0 when its frame is invalid.
__device__ __forceinline__ float decode_sample(const DevStation &S, const uint8_t *__restrict__ buf,
                                               const uint8_t *__restrict__ valid, int64_t g, int band)
{
	int64_t fr = g / S.framesamples;
	int64_t tin = g - fr * S.framesamples;
	if(!valid[fr])
		return 0.0f;
	const uint8_t *pl = buf + fr * S.framebytes + S.header;
	int64_t q = tin * S.nband + band;
	if(S.nbits == 2)
	{
		int64_t bit = q * 2;
		unsigned int byte = __ldg(pl + (bit >> 3));
		return c_lut2[(byte >> (bit & 7)) & 3];
	}
	return c_lut8[__ldg(pl + q)];
}

// In-place radix-2 decimation-in-time FFT of N = 2^L points held in shared
// memory in bit-reversed order; tw holds exp(-2 pi i k / maxN), k < maxN/2.
__device__ void fft_dit_inplace(float2 *x, int L, const float2 *__restrict__ tw, int twscale)
{
	const int N = 1 << L;
	for(int s = 0; s < L; s++)
	{
		const int half = 1 << s;
		const int tstride = (N >> (s + 1)) * twscale;
		for(int q = threadIdx.x; q < (N >> 1); q += blockDim.x)
		{
			int k = q & (half - 1);
			int i = ((q >> s) << (s + 1)) + k;
			int j = i + half;
			float2 w = __ldg(tw + (int64_t)k * tstride);
			float2 a = x[i], b = x[j];
			float2 t = cmul(b, w);
			x[i] = make_float2(a.x + t.x, a.y + t.y);
			x[j] = make_float2(a.x - t.x, a.y - t.y);
		}
		__syncthreads();
	}
}

// One CTA per (FFT, station): Mode::process for every band of the station
// (mode.cpp:845-1308): decode, time-domain fringe rotation (orders 1, 2),
// complex FFT of 2*nchan points, sideband selection, fractional-sample
// rotation (with the post-F fringe phase for order 0).  Output row-major
// spectra [t][row][nchan] per frequency, FP32.
__global__ void __launch_bounds__(256) k_fstage(const DevStation *__restrict__ st, const DevSubintStation *__restrict__ sub,
                                                const DevBand *__restrict__ bands, int maxband,
                                                const DevFreqPlan *__restrict__ plans, const uint8_t *__restrict__ valid,
                                                int64_t valid_stride, const FftParam *__restrict__ params,
                                                const float2 *__restrict__ twiddle, int maxN, int T, int order,
                                                int fractionallofreq, float2 *__restrict__ spec)
{
	extern __shared__ float2 sx[];
	const int t = blockIdx.x, s = blockIdx.y;
	const DevStation &S = st[s];
	const FftParam p = params[(int64_t)s * T + t];
	const int N = S.fftchannels, nchan = S.nchan;
	const int L = 31 - __clz(N);
	const uint8_t *buf = sub[s].buf;
	const uint8_t *vrow = valid + (int64_t)s * valid_stride;
	const int twscale = maxN / N;

	for(int b = 0; b < S.nband; b++)
	{
		const DevBand bd = bands[s * maxband + b];
		if(bd.row < 0)
			continue;
		const DevFreqPlan &pl = plans[bd.freq];
		float2 *out = spec + pl.spec_off + ((int64_t)t * pl.nrow + bd.row) * nchan;
		if(p.status != kFftOk)
		{
			for(int c = threadIdx.x; c < nchan; c += blockDim.x)
				out[c] = make_float2(0.0f, 0.0f);
			continue;
		}
		// fringe phase of sample n in turns: P0 + ... (FP64 reduction of the
		// constant part, FP32 per sample); mode.cpp:790-1051
		const double lo = bd.lofreq;
		const double fraclo = fractionallofreq ? (lo - (int)lo) * (double)p.integerdelay : 0.0;
		float P0 = 0.0f, alpha = 0.0f, beta = 0.0f, gamma = 0.0f, eps = 0.0f;
		const int asl = S.asl;
		if(order == 1)
		{
			double ph0 = lo * p.b + fraclo;
			P0 = (float)(ph0 - floor(ph0));
			alpha = (float)(lo * p.a / N);
		}
		else if(order == 2)
		{
			double X1 = (double)asl / (double)N;
			double ph0 = lo * p.c + fraclo;
			P0 = (float)(ph0 - floor(ph0));
			alpha = (float)(lo * (p.b + p.a * X1) / N);
			beta = (float)(lo * 2.0 * p.a * X1 / N);
			gamma = (float)(lo * p.b * asl / N);
			eps = (float)(lo * p.a * X1 * X1);
		}
		for(int n = threadIdx.x; n < N; n += blockDim.x)
		{
			float v = 0.0f;
			if(n < p.stuck)
				v = decode_sample(S, buf, vrow, (int64_t)p.nearest + n, b);
			float2 z;
			if(order == 0)
				z = make_float2(v, 0.0f);
			else
			{
				float ph;
				if(order == 1)
					ph = P0 + (float)n * alpha;
				else
				{
					int k = n / asl, j = n - k * asl;
					ph = P0 + (float)j * alpha + (float)(k * j) * beta + (float)k * gamma + (float)(k * k) * eps;
				}
				ph -= floorf(ph);
				float sn, cs;
				sincospif(-2.0f * ph, &sn, &cs);
				z = make_float2(v * cs, v * sn);
			}
			sx[__brev(n) >> (32 - L)] = z;
		}
		__syncthreads();
		fft_dit_inplace(sx, L, twiddle, twscale);
		// fractional-sample correction exp(+2 pi i f_c fse), f_c in MHz
		// (mode.cpp:1053-1097, 1279-1286); post-F fringe phase for order 0
		// (mode.cpp:1061-1070)
		const float dfs = (float)(S.bw / nchan * (double)p.fse);
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
			float2 x;
			int ce;
			if(bd.lsb)
			{
				ce = c - nchan;
				if(order == 0)
				{
					float2 y = sx[nchan - c];
					x = make_float2(y.x, -y.y);
				}
				else
					x = sx[nchan + c];
			}
			else
			{
				ce = c;
				x = sx[c];
			}
			float turns = (float)ce * dfs + postf;
			float sn, cs;
			sincospif(2.0f * turns, &sn, &cs);
			out[c] = cmul(x, make_float2(cs, sn));
		}
		__syncthreads();
	}
}

cudaError_t launch_fstage(const DevStation *st, const DevSubintStation *sub, const DevBand *bands, int maxband,
                   const DevFreqPlan *plans, const uint8_t *valid, int64_t valid_stride, const FftParam *params,
                   const float2 *twiddle, int maxN, int S, int T, int order, bool fractionallofreq, int maxfft,
                   float2 *spec, cudaStream_t stream)
{
	size_t smem = (size_t)maxfft * sizeof(float2);
	// the shared-memory limit is a per-device attribute: raised on every call
	// (cheap), so that a launch on any device of the process gets it
	const cudaError_t e = cudaFuncSetAttribute(k_fstage, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
	if(e != cudaSuccess)
		return e;
	dim3 grid(T, S);
	k_fstage<<<grid, 256, smem, stream>>>(st, sub, bands, maxband, plans, valid, valid_stride, params, twiddle, maxN, T,
	                                      order, fractionallofreq ? 1 : 0, spec);
	return cudaGetLastError();
}

// FP32 cross-multiply-accumulate (core.cpp:877-972 with the autocorrelations
// of mode.cpp:1293-1369).  For one frequency, V[i][j] = sum_t X_i X_j^* over
// all input rows is evaluated in 4x4 register tiles (a complex Hermitian
// rank-T update per channel): one warp = one tile pair, 32 channels per CTA.
// Each (output, channel) is owned by one thread, which adds its subint sum
// into the accumulator.
__global__ void __launch_bounds__(256) k_xmac_fp32(const DevFreqPlan *__restrict__ plan, int T, int TC,
                                                   const float2 *__restrict__ spec, float2 *__restrict__ acc)
{
	extern __shared__ float2 sxm[];
	const DevFreqPlan P = *plan;
	constexpr int CB = 32;
	const int c0 = blockIdx.y * CB;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int pairidx = blockIdx.x * 8 + warp;
	const bool active = pairidx < P.npair;
	int ti = 0, tj = 0;
	if(active)
	{
		ti = P.pairs[2 * pairidx];
		tj = P.pairs[2 * pairidx + 1];
	}
	const int nrowpad = P.ntr * kTile;
	const float2 *X = spec + P.spec_off;
	float vr[4][4], vi[4][4];
#pragma unroll
	for(int i = 0; i < 4; i++)
#pragma unroll
		for(int j = 0; j < 4; j++)
		{
			vr[i][j] = 0.0f;
			vi[i][j] = 0.0f;
		}
	for(int t0 = 0; t0 < T; t0 += TC)
	{
		const int tcnt = min(TC, T - t0);
		const int nel = TC * nrowpad * CB;
		for(int e = threadIdx.x; e < nel; e += blockDim.x)
		{
			int c = e % CB;
			int r = (e / CB) % nrowpad;
			int tt = e / (CB * nrowpad);
			float2 v = make_float2(0.0f, 0.0f);
			if(tt < tcnt && r < P.nrow && c0 + c < P.nchan)
				v = X[((int64_t)(t0 + tt) * P.nrow + r) * P.nchan + c0 + c];
			sxm[e] = v;
		}
		__syncthreads();
		if(active)
		{
			for(int tt = 0; tt < tcnt; tt++)
			{
				const float2 *row = sxm + (int64_t)tt * nrowpad * CB;
				float2 a[4], b[4];
#pragma unroll
				for(int i = 0; i < 4; i++)
				{
					a[i] = row[(ti * 4 + i) * CB + lane];
					b[i] = row[(tj * 4 + i) * CB + lane];
				}
#pragma unroll
				for(int i = 0; i < 4; i++)
#pragma unroll
					for(int j = 0; j < 4; j++)
					{
						vr[i][j] = fmaf(a[i].x, b[j].x, fmaf(a[i].y, b[j].y, vr[i][j]));
						vi[i][j] = fmaf(a[i].y, b[j].x, fmaf(-a[i].x, b[j].y, vi[i][j]));
					}
			}
		}
		__syncthreads();
	}
	if(!active)
		return;
	const int c = c0 + lane;
	if(c >= P.nchan)
		return;
#pragma unroll
	for(int i = 0; i < 4; i++)
#pragma unroll
		for(int j = 0; j < 4; j++)
		{
			int ri = ti * 4 + i, rj = tj * 4 + j;
			if(ri >= P.nrow || rj >= P.nrow || (ti == tj && i > j))
				continue;
			int dA = P.destA[ri * P.nrow + rj];
			int dB = P.destB[ri * P.nrow + rj];
			if(dA >= 0)
			{
				float2 *d = acc + P.acc_off + (int64_t)dA * P.nchan + c;
				float2 o = *d;
				*d = make_float2(o.x + vr[i][j], o.y + vi[i][j]);
			}
			if(dB >= 0)
			{
				float2 *d = acc + P.acc_off + (int64_t)dB * P.nchan + c;
				float2 o = *d;
				*d = make_float2(o.x + vr[i][j], o.y - vi[i][j]);
			}
		}
}

void launch_xmac_fp32(const DevFreqPlan &plan, const DevFreqPlan *dplan, int T, const float2 *spec, float2 *acc,
                      cudaStream_t stream)
{
	constexpr int CB = 32;
	const int nrowpad = plan.ntr * kTile;
	int TC = (96 * 1024) / (nrowpad * CB * (int)sizeof(float2));
	if(TC > 32) TC = 32;
	if(TC < 1) TC = 1;
	size_t smem = (size_t)TC * nrowpad * CB * sizeof(float2);
	// per-device attribute: raised on every call
	if(cudaFuncSetAttribute(k_xmac_fp32, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024) != cudaSuccess)
		return;
	dim3 grid((plan.npair + 7) / 8, (plan.nchan + CB - 1) / CB);
	k_xmac_fp32<<<grid, 256, smem, stream>>>(dplan, T, TC, spec, acc);
}

// Baseline weights sum_t w1*w2 (core.cpp:998-1045) and autocorrelation
// weights sum_t w (mode.cpp:1304-1307), each as a sequential float sum in FFT
// order, added to the running totals (core.cpp:1068-1086, 1310-1363).
// Baseline and autocorrelation weights of one subint: the float sums of
// w1(t) * w2(t) (baseline) and of w(t) over valid FFTs (autocorrelation), added
// in FFT order as Core does.  One warp per weight: the lanes load and multiply
// 256 FFTs at a time in parallel, then lane 0 adds them in order (adding 0 for
// an invalid FFT leaves a non-negative float sum unchanged).
// INTERLACEDVDIF stations weigh each band by its own data weight
// (Mode::getDataWeight, mode.h:168, mode.cpp:1300-1303).
__global__ void k_weights(const DevBWeight *__restrict__ bw, int nbw, const DevACWeight *__restrict__ acw, int nacw,
                          const FftParam *__restrict__ params, const float *__restrict__ pbw, int nbm,
                          const DevStation *__restrict__ st, int T, float *__restrict__ bwacc,
                          float *__restrict__ acwacc)
{
	__shared__ float buf[4][256];
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int k = blockIdx.x * 4 + w;
	if(k >= nbw + nacw)
		return;
	const bool isb = k < nbw;
	const FftParam *p1 = params + (int64_t)(isb ? bw[k].s1 : acw[k - nbw].s) * T;
	const FftParam *p2 = params + (int64_t)(isb ? bw[k].s2 : 0) * T;
	const int sa = isb ? bw[k].s1 : acw[k - nbw].s, sb = isb ? bw[k].s2 : sa;
	const int ba = isb ? bw[k].b1 : acw[k - nbw].band, bb = isb ? bw[k].b2 : -1;
	const float *wa = (pbw && st[sa].mux) ? pbw + (int64_t)sa * T * nbm + ba : nullptr;
	const float *wb = (pbw && st[sb].mux && bb >= 0) ? pbw + (int64_t)sb * T * nbm + bb : nullptr;
	float sum = 0.0f;
	for(int t0 = 0; t0 < T; t0 += 256)
	{
		const int n = min(256, T - t0);
		for(int j = lane; j < n; j += 32)
		{
			const int t = t0 + j;
			float v;
			const float w1 = wa ? wa[(int64_t)t * nbm] : p1[t].weight;
			if(isb)
				v = __fmul_rn(w1, wb ? wb[(int64_t)t * nbm] : p2[t].weight);
			else if(p1[t].status != kFftOk)
				v = 0.0f;
			else
				v = w1;
			buf[w][j] = v;
		}
		__syncwarp();
		if(lane == 0)
			for(int j = 0; j < n; j++)
				sum = __fadd_rn(sum, buf[w][j]);
		__syncwarp();
	}
	if(lane == 0)
	{
		if(isb)
			bwacc[k] = __fadd_rn(bwacc[k], sum);
		else
			acwacc[k - nbw] = __fadd_rn(acwacc[k - nbw], sum);
	}
}

void launch_weights(const DevBWeight *bw, int nbw, const DevACWeight *acw, int nacw, const FftParam *params,
                    const float *pbw, int nbm, const DevStation *st, int T, float *bwacc, float *acwacc,
                    cudaStream_t stream)
{
	int n = nbw + nacw;
	if(n == 0)
		return;
	k_weights<<<(n + 3) / 4, 128, 0, stream>>>(bw, nbw, acw, nacw, params, pbw, nbm, st, T, bwacc, acwacc);
}

// Core-result assembly (core.cpp:1774-1802 channel averaging, 1266-1363):
// accumulators -> [freq][baseline][product][nchan/avg], autocorrelations,
// and the float weight slots.
__global__ void k_finalise(const DevOutMap *__restrict__ om, const float2 *__restrict__ acc, float2 *__restrict__ core)
{
	const DevOutMap m = om[blockIdx.x];
	const int nout = m.nchan / m.avg;
	for(int co = threadIdx.x; co < nout; co += blockDim.x)
	{
		float2 v = make_float2(0.0f, 0.0f);
		if(m.acc >= 0)
		{
			if(m.avg == 1)
				v = acc[m.acc + (int64_t)co * m.cstride];
			else
			{
				float sr = 0.0f, si = 0.0f;
				for(int k = 0; k < m.avg; k++)
				{
					float2 a = acc[m.acc + ((int64_t)co * m.avg + k) * m.cstride];
					sr += a.x;
					si += a.y;
				}
				v = make_float2(sr / m.avg, si / m.avg);
			}
		}
		core[m.core + co] = v;
	}
}

__global__ void k_finalise_weights(const DevBWeight *__restrict__ bw, int nbw, const float *__restrict__ bwacc,
                                   const DevACWeight *__restrict__ acw, int nacw, const float *__restrict__ acwacc,
                                   float *__restrict__ corefloat)
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if(k < nbw)
		corefloat[bw[k].dst] = bwacc[k];
	else if(k < nbw + nacw)
		corefloat[acw[k - nbw].dst] = acwacc[k - nbw];
}

void launch_finalise(const DevOutMap *om, int nom, int maxout, const float2 *acc, const DevBWeight *bw, int nbw,
                     const float *bwacc, const DevACWeight *acw, int nacw, const float *acwacc, float2 *core,
                     int64_t corelen, cudaStream_t stream)
{
	(void)maxout;
	cudaMemsetAsync(core, 0, sizeof(float2) * corelen, stream);
	if(nom > 0)
		k_finalise<<<nom, 256, 0, stream>>>(om, acc, core);
	int n = nbw + nacw;
	if(n > 0)
		k_finalise_weights<<<(n + 127) / 128, 128, 0, stream>>>(bw, nbw, bwacc, acw, nacw, acwacc, (float *)core);
}

// Stand-alone decode with mark5_unpack_with_offset's contract
// (mark5_stream_unpacker.c:129-147): one CTA; frame validity first, then the
// good-sample count (with the 8-bit 2/4-channel blank semantics), then the
// samples.
__global__ void k_vdif_unpack(const uint8_t *__restrict__ data, int64_t nbytes, int payload, int header, int nchan,
                              int nbits, int64_t offsetsamples, int nsamp, float *__restrict__ out, int *good)
{
	extern __shared__ uint8_t fvalid[];
	__shared__ int firstblank;
	__shared__ int goodcount;
	const int64_t framebytes = payload + header;
	const int64_t fs = (int64_t)payload * 8 / (nchan * nbits);
	const int64_t f0 = offsetsamples / fs, f1 = (offsetsamples + nsamp - 1) / fs;
	const int nf = (int)(f1 - f0 + 1);
	const uint64_t FILL = 0x1122334411223344ULL;
	for(int k = threadIdx.x; k < nf; k += blockDim.x)
	{
		int64_t fr = f0 + k;
		uint8_t v = 0;
		if((fr + 1) * framebytes <= nbytes)
		{
			const uint8_t *f = data + fr * framebytes;
			uint32_t w0 = *(const uint32_t *)f, w2 = *(const uint32_t *)(f + 8);
			uint64_t first = *(const uint64_t *)(f + header);
			uint64_t last = *(const uint64_t *)(f + header + (payload / 8 - 1) * 8);
			v = (w2 != 0) && !((w0 >> 31) & 1) && first != FILL && last != FILL;
		}
		fvalid[k] = v;
	}
	__syncthreads();
	const bool sticky = nbits == 8 && (nchan == 2 || nchan == 4);
	if(threadIdx.x == 0)
	{
		int fb = nsamp, cnt = 0;
		for(int k = 0; k < nf; k++)
		{
			int64_t a = (f0 + k) * fs - offsetsamples, b = a + fs;
			if(a < 0) a = 0;
			if(b > nsamp) b = nsamp;
			if(!fvalid[k])
			{
				if(sticky && fb == nsamp) fb = (int)a;
				continue;
			}
			if(sticky && fb < nsamp) continue;
			cnt += (int)(b - a);
		}
		firstblank = sticky ? fb : nsamp;
		goodcount = cnt;
	}
	__syncthreads();
	for(int o = threadIdx.x; o < nsamp; o += blockDim.x)
	{
		int64_t g = offsetsamples + o;
		int64_t fr = g / fs, tin = g - fr * fs;
		bool v = fvalid[fr - f0] && o < firstblank;
		const uint8_t *pl = data + fr * framebytes + header;
		for(int c = 0; c < nchan; c++)
		{
			float val = 0.0f;
			if(v)
			{
				int64_t q = tin * nchan + c;
				if(nbits == 2)
				{
					int64_t bit = q * 2;
					val = c_lut2[(pl[bit >> 3] >> (bit & 7)) & 3];
				}
				else
					val = c_lut8[pl[q]];
			}
			out[(int64_t)c * nsamp + o] = val;
		}
	}
	if(threadIdx.x == 0)
		*good = goodcount;
}

void launch_vdif_unpack(const uint8_t *data, int64_t nbytes, int payload, int header, int nchan, int nbits,
                        int64_t offsetsamples, int nsamp, float *out, int *good, cudaStream_t stream)
{
	const int64_t fs = (int64_t)payload * 8 / (nchan * nbits);
	const int nf = (int)((offsetsamples + nsamp - 1) / fs - offsetsamples / fs + 1);
	k_vdif_unpack<<<1, 256, nf, stream>>>(data, nbytes, payload, header, nchan, nbits, offsetsamples, nsamp, out, good);
}

// ---------------------------------------------------------------- zoom bands
// A zoom band's spectra are the channels [choff, choff + nchan) of its parent
// band's (mode.cpp:169-208): one CTA per (8 FFTs, zoom row) copies them into
// the zoom frequency's own spectra rows, FP32 [t][row][chan] (float2) or the
// tensor-core form's blocked [t][block][row][tcb] (bf16x2 as uint32).  Each
// thread finds its channel's block and offset once and steps them.
constexpr int kZoomTimes = 8;

// Position of channel c in a spectra row: block and offset in it (blocks of
// tcb channels; one block of nchan in the FP32 form), advanced by a constant
// step without divisions.
struct ChanPos {
	int blk, off, dblk, doff, width;
	__device__ __forceinline__ ChanPos(int c, int step, int tcb, int nchan)
	{
		width = tcb ? tcb : nchan;
		blk = c / width;
		off = c - blk * width;
		dblk = step / width;
		doff = step - dblk * width;
	}
	__device__ __forceinline__ void advance()
	{
		blk += dblk;
		off += doff;
		if(off >= width)
		{
			off -= width;
			blk++;
		}
	}
};

// element (t, row, block 0, offset 0) and the distance between blocks
__device__ __forceinline__ int64_t row_base(const DevFreqPlan &p, int t, int row)
{
	if(p.tcb == 0)
		return p.spec_off + ((int64_t)t * p.nrow + row) * p.nchan;
	return p.spec_off + ((int64_t)t * p.tnblk * p.nrow + row) * p.tcb;
}

__device__ __forceinline__ int64_t block_stride(const DevFreqPlan &p) { return p.tcb ? (int64_t)p.nrow * p.tcb : 0; }

template <typename V>
__global__ void __launch_bounds__(256) k_zoom_gather(const DevZoomCopy *__restrict__ zc,
                                                     const DevFreqPlan *__restrict__ plans, int T,
                                                     V *__restrict__ spec)
{
	const DevZoomCopy z = zc[blockIdx.y];
	const DevFreqPlan src = plans[z.src_plan], dst = plans[z.dst_plan];
	const int t0 = blockIdx.x * kZoomTimes, t1 = min(T, t0 + kZoomTimes);
	const int64_t sbs = block_stride(src), dbs = block_stride(dst);
	const ChanPos sp0(z.choff + (int)threadIdx.x, blockDim.x, src.tcb, src.nchan);
	const ChanPos dp0((int)threadIdx.x, blockDim.x, dst.tcb, dst.nchan);
	const int64_t sts = row_base(src, 1, z.src_row) - row_base(src, 0, z.src_row);
	const int64_t dts = row_base(dst, 1, z.dst_row) - row_base(dst, 0, z.dst_row);
	int64_t sb = row_base(src, t0, z.src_row), db = row_base(dst, t0, z.dst_row);
	for(int t = t0; t < t1; t++, sb += sts, db += dts)
	{
		ChanPos sp = sp0, dp = dp0;
		for(int c = threadIdx.x; c < z.nchan; c += blockDim.x)
		{
			spec[db + dp.blk * dbs + dp.off] = spec[sb + sp.blk * sbs + sp.off];
			sp.advance();
			dp.advance();
		}
	}
}

void launch_zoom_gather(const DevZoomCopy *zc, int nzc, const DevFreqPlan *plans, int T, bool tc, void *spec,
                        cudaStream_t stream)
{
	if(nzc <= 0 || T <= 0)
		return;
	const dim3 grid((T + kZoomTimes - 1) / kZoomTimes, nzc);
	if(tc)
		k_zoom_gather<uint32_t><<<grid, 256, 0, stream>>>(zc, plans, T, (uint32_t *)spec);
	else
		k_zoom_gather<float2><<<grid, 256, 0, stream>>>(zc, plans, T, (float2 *)spec);
}

// 8-bit levels (b - 128) / 3.3 (format_vdif.c:122) into the current
// device's constant table; pageable source, so the copy has been taken when
// this returns
cudaError_t upload_lut8(cudaStream_t stream)
{
	float lut[256];
	for(int b = 0; b < 256; b++)
		lut[b] = (float)((b - 128) / 3.3);
	return cudaMemcpyToSymbolAsync(c_lut8, lut, sizeof(lut), 0, cudaMemcpyHostToDevice, stream);
}

}  // namespace fxb
