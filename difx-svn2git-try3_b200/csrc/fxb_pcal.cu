// Phase-cal extraction (mode.cpp:773-787, pcal.cpp:927-1105, core.cpp:1124-1150).
//
// The reference's implicit-shift extractor adds every unpacked sample of
// every valid FFT window into bin (sample number in the data second) mod N
// and, at the end of the subint, takes a length-N DFT whose bins at the tone
// frequencies are the tones.  The DFT is linear, so the device keeps the bins
// summed over every subint of the integration (FP64, one slice per chunk of
// FFTs) and takes the DFT once, when the core result is read.
//
// k_pcal_bin: one CTA per (chunk of FFTs, group of a station's bands with the
// same bin count N).  Samples are decoded as the F stage decodes them (zero
// outside valid frames and past the window's blanking point).  Each thread
// owns bins and sums their samples in a fixed order -- with N below the CTA
// width, Q = 256 / N lanes split a bin's samples and are added in lane
// order -- and each CTA adds its bins, without atomics, into its chunk's own
// slice of the FP64 bins, so that the result does not depend on scheduling.
// k_pcal_final: one CTA per band, the chunks summed in order and the DFT at
// the tone bins, in FP64.

#include <algorithm>

#include "fxb_kernels.h"

namespace fxb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float level2(uint32_t code)
{
	// 2-bit code -> {-HiMag, -1, +1, +HiMag} (format_vdif.c:78)
	const float mag = ((code ^ (code >> 1)) & 1u) ? 1.0f : 3.3359f;
	return (code & 2u) ? mag : -mag;
}

// Decoder of one station's samples in one FFT window: sample n of the window
// for every band of the group, 0 outside valid frames and past the blanking
// point.  Samples are visited with a constant stride, so the frame and the
// time within it advance without divisions.
struct Window {
	const uint8_t *buf, *vrow;
	int64_t valid_stride;
	uint32_t fa, fs, framebytes, header, bpt, nbits, mask;
	int stuck;
};

// Adds samples n0, n0 + step, ... (< L) of the window, which starts so
// samples into frame fa, to acc[band].
template <int NB>
__device__ __forceinline__ void sum_samples_from(const Window &w, const DevPcalGroup &g, const float *lut8,
                                                 uint32_t so, int n0, int step, int L, float (&acc)[NB])
{
	if(n0 >= L)
		return;
	const uint32_t x0 = so + (uint32_t)n0;
	uint32_t kf = x0 / w.fs, tin = x0 - kf * w.fs;
	for(int n = n0; n < L; n += step)
	{
		const int64_t fr = (int64_t)w.fa + kf;
		if(n < w.stuck && fr < w.valid_stride && w.vrow[fr] != 0)
		{
			const uint32_t *wp = (const uint32_t *)(w.buf + fr * w.framebytes + w.header);
#pragma unroll
			for(int j = 0; j < NB; j++)
				if(j < g.nb)
				{
					const uint32_t bit = tin * w.bpt + (uint32_t)g.band[j] * w.nbits;
					const uint32_t code = (__ldg(wp + (bit >> 5)) >> (bit & 31u)) & w.mask;
					acc[j] += w.nbits == 2 ? level2(code) : lut8[code];
				}
		}
		tin += (uint32_t)step;
		while(tin >= w.fs)
		{
			tin -= w.fs;
			kf++;
		}
	}
}

__global__ void __launch_bounds__(kThreads) k_pcal_bin(const DevPcalGroup *__restrict__ groups,
                                                      const DevStation *__restrict__ st,
                                                      const DevSubintStation *__restrict__ sub,
                                                      const FftParam *__restrict__ params,
                                                      const uint8_t *__restrict__ valid, int64_t valid_stride, int T,
                                                      int tpc, int64_t chunk_stride, double *__restrict__ bins)
{
	extern __shared__ float sm[];              // bins [nb][N], then (N < 256) lane partials [Q][nb][N]
	__shared__ float lut8[256];
	const DevPcalGroup &g = groups[blockIdx.y];
	const int s = g.station, nb = g.nb, N = g.nbins;
	const DevStation &S = st[s];
	const int tid = threadIdx.x;
	const int Q = N >= kThreads ? 1 : kThreads / N;
	float *part = sm + nb * N;
	for(int i = tid; i < nb * N; i += kThreads)
		sm[i] = 0.0f;
	if(S.nbits == 8)
		for(int i = tid; i < 256; i += kThreads)
			lut8[i] = (float)((i - 128) / 3.3);      // format_vdif.c:122
	__syncthreads();
	Window w;
	w.buf = sub[s].buf;
	w.vrow = valid + (int64_t)s * valid_stride;
	w.valid_stride = valid_stride;
	w.fs = (uint32_t)S.framesamples;
	w.framebytes = (uint32_t)S.framebytes;
	w.header = (uint32_t)S.header;
	w.nbits = (uint32_t)S.nbits;
	w.bpt = (uint32_t)(S.nbits * S.nband);
	w.mask = (1u << S.nbits) - 1u;
	const int64_t datasamples = (int)(sub[s].datans / (S.sampletime * 1e3) + 0.5);   // Mode::setData
	const int L = S.fftchannels;
	const int t1 = min(T, (int)(blockIdx.x + 1) * tpc);
	for(int t = blockIdx.x * tpc; t < t1; t++)
	{
		const FftParam &p = params[(int64_t)s * T + t];
		if(p.status != kFftOk)
			continue;                               // the same for the whole CTA
		const int r = (int)((datasamples + p.nearest) % N);
		const uint32_t g0 = (uint32_t)p.nearest;
		w.fa = g0 / w.fs;
		w.stuck = p.stuck;
		const uint32_t so = g0 - w.fa * w.fs;
		if(N < kThreads)
		{
			const int q = tid / N, m = tid - q * N;
			if(q < Q)
			{
				float acc[kPcalGroupBands];
#pragma unroll
				for(int j = 0; j < kPcalGroupBands; j++)
					acc[j] = 0.0f;
				int n0 = m - r;
				if(n0 < 0)
					n0 += N;
				sum_samples_from(w, g, lut8, so, n0 + q * N, Q * N, L, acc);
#pragma unroll
				for(int j = 0; j < kPcalGroupBands; j++)
					if(j < nb)
						part[(q * nb + j) * N + m] = acc[j];
			}
			__syncthreads();
			for(int i = tid; i < nb * N; i += kThreads)
			{
				const int j = i / N, m2 = i - j * N;
				float v = 0.0f;
				for(int q2 = 0; q2 < Q; q2++)
					v += part[(q2 * nb + j) * N + m2];
				sm[i] += v;
			}
			__syncthreads();
		}
		else
			for(int m = tid; m < N; m += kThreads)
			{
				float acc[kPcalGroupBands];
#pragma unroll
				for(int j = 0; j < kPcalGroupBands; j++)
					acc[j] = 0.0f;
				int n0 = m - r;
				if(n0 < 0)
					n0 += N;
				sum_samples_from(w, g, lut8, so, n0, N, L, acc);
#pragma unroll
				for(int j = 0; j < kPcalGroupBands; j++)
					if(j < nb)
						sm[j * N + m] += acc[j];       // bin m belongs to this thread alone
			}
	}
	__syncthreads();
	double *dst = bins + (int64_t)blockIdx.x * chunk_stride;
	for(int i = tid; i < nb * N; i += kThreads)
	{
		const int j = i / N;
		dst[g.bin_off[j] + (i - j * N)] += (double)sm[i];
	}
}

__global__ void __launch_bounds__(kThreads) k_pcal_final(const DevPcalBand *__restrict__ bands, int nchunk,
                                                        int64_t chunk_stride, const double *__restrict__ bins,
                                                        float2 *__restrict__ core)
{
	__shared__ double red[2][kThreads / 32];
	const DevPcalBand b = bands[blockIdx.x];
	const int N = b.nbins;
	for(int k = 0; k < b.ntones; k++)
	{
		const int64_t idx = (int64_t)b.first + (int64_t)k * b.step;
		double re = 0.0, im = 0.0;
		if(N > 0 && idx < N)
			for(int m = threadIdx.x; m < N; m += kThreads)
			{
				// X[idx] = sum_m Z[m] exp(-2 pi i idx m / N), the angle reduced exactly
				double sn, cs;
				sincospi(-2.0 * (double)((idx * m) % N) / (double)N, &sn, &cs);
				double z = 0.0;
				for(int c = 0; c < nchunk; c++)          // the chunks' bins, in chunk order
					z += bins[c * chunk_stride + b.bin_off + m];
				re += z * cs;
				im += z * sn;
			}
		for(int o = 16; o > 0; o >>= 1)
		{
			re += __shfl_xor_sync(0xffffffffu, re, o);
			im += __shfl_xor_sync(0xffffffffu, im, o);
		}
		if((threadIdx.x & 31) == 0)
		{
			red[0][threadIdx.x >> 5] = re;
			red[1][threadIdx.x >> 5] = im;
		}
		__syncthreads();
		if(threadIdx.x == 0)
		{
			double sr = 0.0, si = 0.0;
			for(int w = 0; w < kThreads / 32; w++)
			{
				sr += red[0][w];
				si += red[1][w];
			}
			core[b.core + k] = make_float2((float)sr, (float)si);
		}
		__syncthreads();
	}
}

}  // namespace

size_t pcal_group_smem(const DevPcalGroup &g)
{
	const size_t lanes = g.nbins >= kThreads ? 0 : (size_t)(kThreads / g.nbins);
	return (size_t)g.nb * g.nbins * (1 + lanes) * sizeof(float);
}

void launch_pcal_bin(const DevPcalGroup *groups, int ngroups, size_t smem, int nchunk, const DevStation *st,
                     const DevSubintStation *sub, const FftParam *params, const uint8_t *valid, int64_t valid_stride,
                     int T, int64_t chunk_stride, double *bins, cudaStream_t stream)
{
	if(ngroups <= 0)
		return;
	const int tpc = (T + nchunk - 1) / nchunk;
	const dim3 grid((T + tpc - 1) / tpc, ngroups);
	k_pcal_bin<<<grid, kThreads, smem, stream>>>(groups, st, sub, params, valid, valid_stride, T, tpc, chunk_stride,
	                                            bins);
}

cudaError_t pcal_init(size_t smem)
{
	return cudaFuncSetAttribute(k_pcal_bin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

void launch_pcal_final(const DevPcalBand *bands, int nbands, int nchunk, int64_t chunk_stride, const double *bins,
                       float2 *core, cudaStream_t stream)
{
	if(nbands > 0)
		k_pcal_final<<<nbands, kThreads, 0, stream>>>(bands, nchunk, chunk_stride, bins, core);
}

}  // namespace fxb
