// Phase-cal extraction (mode.cpp:773-787, pcal.cpp:494-705, 927-1105,
// core.cpp:1124-1150).
//
// The reference's implicit-shift extractor adds every unpacked sample of
// every valid FFT window into bin (sample number in the data second) mod N
// and, at the end of the subint, takes a length-N DFT whose bins at the tone
// frequencies are the tones; the shifting extractor first rotates each sample
// by exp(-2 pi i offset a / fs) and folds into complex bins.  The DFT is linear, so the device keeps the bins
// summed over every subint of the integration (FP64, one slice per chunk of
// FFTs) and takes the DFT once, when the core result is read.
//
// k_pcal_bin: CTAs over (chunk of FFTs, block of bins, group of a station's
// bands with the same bin count N).  Samples are decoded as the F stage
// decodes them (zero outside valid frames and past the window's blanking
// point).  Every bin is summed in a fixed order and each CTA adds its bins,
// without atomics, into its chunk's own slice of the FP64 bins, so that the
// result does not depend on scheduling.
// k_pcal_final: one CTA per band, the chunks summed in order and the DFT at
// the tone bins, in FP64.

#include <algorithm>

#include "fxb_kernels.h"

namespace fxb {

namespace {

constexpr int kThreads = 256;

// Per-thread sums of one bin over samples: SWAR lane counters (2-bit, 16
// bands to a word) or per-band float sums.
template <int NBITS, bool ONEWORD, bool SWAR, bool SHIFT>
struct BinSum {
	uint32_t le = 0, lo = 0, he = 0, ho = 0;
	int nv = 0;
	float acc[kPcalGroupBands];
	float acci[SHIFT ? kPcalGroupBands : 1];   // imaginary parts (shifting extractor)
	__device__ __forceinline__ BinSum()
	{
#pragma unroll
		for(int j = 0; j < kPcalGroupBands; j++)
			acc[j] = 0.0f;
#pragma unroll
		for(int j = 0; j < (SHIFT ? kPcalGroupBands : 1); j++)
			acci[j] = 0.0f;
	}
	__device__ __forceinline__ void flush(const uint32_t (&boff)[kPcalGroupBands], int nb)
	{
#pragma unroll
		for(int j = 0; j < kPcalGroupBands; j++)
			if(j < nb)
			{
				const uint32_t f = boff[j] >> 1, sh = 4u * (f >> 1);
				const int ca = (int)((((f & 1u) ? ho : he) >> sh) & 15u);
				const int cb = (int)((((f & 1u) ? lo : le) >> sh) & 15u);
				acc[j] += 3.3359f * (float)(ca + cb - nv) + (float)(ca - cb);
			}
		le = lo = he = ho = 0u;
		nv = 0;
	}
	// one sample: its word (ONEWORD) or frame words, the bit of its time and
	// (SHIFT) the rotator exp(-2 pi i offset a / fs) of its sample number a
	__device__ __forceinline__ void add(uint32_t word, const uint32_t *wp, uint32_t tbit,
	                                    const uint32_t (&boff)[kPcalGroupBands], int nb, const float *lut, float rc = 1.0f,
	                                    float rs = 0.0f)
	{
		if(SWAR)
		{
			le += word & 0x11111111u;
			lo += (word >> 2) & 0x11111111u;
			he += (word >> 1) & 0x11111111u;
			ho += (word >> 3) & 0x11111111u;
			if(++nv == 15)
				flush(boff, nb);
		}
		else
		{
#pragma unroll
			for(int j = 0; j < kPcalGroupBands; j++)
				if(j < nb)
				{
					const uint32_t bit = tbit + boff[j];
					const uint32_t wd = ONEWORD ? word : __ldg(wp + (bit >> 5));
					const float v = lut[(wd >> (bit & 31u)) & ((1u << NBITS) - 1u)];
					if(SHIFT)
					{
						acc[j] += v * rc;
						acci[SHIFT ? j : 0] += v * rs;
					}
					else
						acc[j] += v;
				}
		}
	}
};

// One thread per (bin, lane) of a station's group: the thread walks its
// lane's FFT windows of the CTA's chunk in order and sums every sample that
// falls into its bin, all bands of a word at once.  Bin counts below the CTA
// width give each bin Q = 256 / N lanes, which take every Q-th window of the
// chunk and are added in lane order; larger counts give each bin one lane and
// spread the bins over CTAs.  The CTA adds its sums, without atomics, into
// its chunk's slice of the FP64 bins.  The samples of eight windows are loaded
// before any is used.
template <int NBITS, bool ONEWORD, bool SWAR, bool SHIFT>
__global__ void __launch_bounds__(kThreads) k_pcal_bin(const DevPcalGroup *__restrict__ groups,
                                                      const DevStation *__restrict__ st,
                                                      const DevSubintStation *__restrict__ sub,
                                                      const FftParam *__restrict__ params,
                                                      const uint8_t *__restrict__ valid, int64_t valid_stride, int T,
                                                      int tpc, int64_t chunk_stride, double *__restrict__ bins)
{
	extern __shared__ int4 ftab[];             // per FFT of the chunk: residue of its first sample, first frame, offset, blanking;
	                                           // then the rotator phase of its first sample (SHIFT), then lane sums
	__shared__ float lut[1 << NBITS];
	const DevPcalGroup &g = groups[blockIdx.y];
	const int s = g.station, nb = g.nb, N = g.nbins;
	const DevStation &S = st[s];
	const int tid = threadIdx.x;
	const int L = S.fftchannels;
	const uint32_t fs = (uint32_t)S.framesamples;
	// CTAs of bins per chunk: the launch's (gridDim.x / chunks) for its
	// largest bin count; blocks past this group's bins have nothing to do
	const int nbb = gridDim.x / ((T + tpc - 1) / tpc);
	const int chunk = blockIdx.x / nbb, bb = blockIdx.x - chunk * nbb;
	if(bb * kThreads >= N)
		return;
	const int t0 = chunk * tpc, t1 = min(T, t0 + tpc);
	const int64_t datasamples = (int)(sub[s].datans / (S.sampletime * 1e3) + 0.5);   // Mode::setData
	int32_t *fph = reinterpret_cast<int32_t *>(ftab + tpc);   // (offset x first sample) mod fs
	const int64_t fsi = g.fs, off = g.shift;
	for(int t = t0 + tid; t < t1; t += kThreads)
	{
		const FftParam &p = params[(int64_t)s * T + t];
		int4 e = make_int4(-1, 0, 0, 0);
		if(p.status == kFftOk)
		{
			const uint32_t g0 = (uint32_t)p.nearest;
			e.x = (int)((datasamples + p.nearest) % N);
			e.y = (int)(g0 / fs);
			e.z = (int)(g0 - (uint32_t)e.y * fs);
			e.w = p.stuck;
			if(SHIFT)
				fph[t - t0] = (int32_t)((off * ((datasamples + p.nearest) % fsi)) % fsi);
		}
		ftab[t - t0] = e;
	}
	for(int i = tid; i < (1 << NBITS); i += kThreads)
		lut[i] = NBITS == 2 ? ((i & 2) ? 1.0f : -1.0f) * (((i ^ (i >> 1)) & 1) ? 1.0f : 3.3359f)   // format_vdif.c:78
		                    : (float)((i - 128) / 3.3);                                              // format_vdif.c:122
	__syncthreads();
	const int Q = N < kThreads ? kThreads / N : 1;
	const int q = N < kThreads ? tid / N : 0;
	const int m = N < kThreads ? tid - q * N : bb * kThreads + tid;
	const bool active = q < Q && m < N;
	uint32_t boff[kPcalGroupBands];
#pragma unroll
	for(int j = 0; j < kPcalGroupBands; j++)
		boff[j] = j < nb ? (uint32_t)g.band[j] * NBITS : 0u;
	BinSum<NBITS, ONEWORD, SWAR, SHIFT> sum;
	// rotator phase step between a bin's samples of one window (N apart)
	const int64_t dph = SHIFT ? (off * N) % fsi : 0;
	if(active)
	{
		const uint8_t *buf = sub[s].buf;
		const uint8_t *vrow = valid + (int64_t)s * valid_stride;
		const uint32_t framebytes = (uint32_t)S.framebytes, header = (uint32_t)S.header,
		               bpt = (uint32_t)(NBITS * S.nband);
		const int nt = t1 - t0;
		// the next sample of bin m: window t (relative to t0), sample n of it
		// (n = L: not yet found in window t)
		int t = q, n = L;
		int64_t ph = 0;                        // rotator phase (x fs) of sample n of window t
		constexpr int K = 8;
		while(true)
		{
			uint32_t word[K], tbit[K];
			const uint32_t *wp[K];
			bool ok[K];
			int32_t phk[SHIFT ? K : 1];
#pragma unroll
			for(int k = 0; k < K; k++)
			{
				ok[k] = false;
				word[k] = tbit[k] = 0u;
				wp[k] = nullptr;
				while(t < nt && n >= L)
				{
					const int4 e = ftab[t];
					if(e.x >= 0)
					{
						n = m - e.x;
						if(n < 0)
							n += N;
					}
					if(e.x < 0 || n >= L)
					{
						t += Q;
						n = L;
					}
					else if(SHIFT)
						ph = (fph[t] + (off * n) % fsi) % fsi;
				}
				if(t < nt)
				{
					const int4 e = ftab[t];
					if(SHIFT)
						phk[SHIFT ? k : 0] = (int32_t)ph;
					uint32_t x = (uint32_t)e.z + (uint32_t)n, kf = 0;
					while(x >= fs)
					{
						x -= fs;
						kf++;
					}
					const int64_t fr = (int64_t)e.y + kf;
					ok[k] = n < e.w && fr < valid_stride && vrow[fr] != 0;
					tbit[k] = x * bpt;
					wp[k] = (const uint32_t *)(buf + fr * framebytes + header);
					if(ok[k] && ONEWORD)
						word[k] = __ldg(wp[k] + (tbit[k] >> 5));
					n += N;
					if(SHIFT)
					{
						ph += dph;
						if(ph >= fsi)
							ph -= fsi;
					}
					if(n >= L)
					{
						t += Q;
						n = L;
					}
				}
			}
#pragma unroll
			for(int k = 0; k < K; k++)
				if(ok[k])
				{
					float rs = 0.0f, rc = 1.0f;
					if(SHIFT)
						sincospif(-2.0f * ((float)phk[SHIFT ? k : 0] / (float)fsi), &rs, &rc);
					sum.add(word[k], wp[k], tbit[k], boff, nb, lut, rc, rs);
				}
			if(t >= nt)
				break;
		}
		if(SWAR && sum.nv)
			sum.flush(boff, nb);
	}
	double *dst = bins + (int64_t)chunk * chunk_stride;
	constexpr int C = SHIFT ? 2 : 1;          // doubles per bin
	if(Q == 1)
	{
		if(active)
#pragma unroll
			for(int j = 0; j < kPcalGroupBands; j++)
				if(j < nb)
				{
					dst[g.bin_off[j] + C * m] += (double)sum.acc[j];
					if(SHIFT)
						dst[g.bin_off[j] + C * m + 1] += (double)sum.acci[SHIFT ? j : 0];
				}
		return;
	}
	// lanes of a bin, added in lane order
	float *part = reinterpret_cast<float *>(fph + tpc);    // [Q][nb][N][C]
	if(active)
#pragma unroll
		for(int j = 0; j < kPcalGroupBands; j++)
			if(j < nb)
			{
				part[((q * nb + j) * N + m) * C] = sum.acc[j];
				if(SHIFT)
					part[((q * nb + j) * N + m) * C + 1] = sum.acci[SHIFT ? j : 0];
			}
	__syncthreads();
	for(int i = tid; i < nb * N; i += kThreads)
	{
		const int j = i / N, mm = i - j * N;
		float v = 0.0f, vi = 0.0f;
		for(int q2 = 0; q2 < Q; q2++)
		{
			v += part[((q2 * nb + j) * N + mm) * C];
			if(SHIFT)
				vi += part[((q2 * nb + j) * N + mm) * C + 1];
		}
		dst[g.bin_off[j] + C * mm] += (double)v;
		if(SHIFT)
			dst[g.bin_off[j] + C * mm + 1] += (double)vi;
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
				double z = 0.0, zi = 0.0;
				for(int c = 0; c < nchunk; c++)          // the chunks' bins, in chunk order
				{
					if(b.shift)
					{
						z += bins[c * chunk_stride + b.bin_off + 2 * m];
						zi += bins[c * chunk_stride + b.bin_off + 2 * m + 1];
					}
					else
						z += bins[c * chunk_stride + b.bin_off + m];
				}
				re += z * cs - zi * sn;
				im += z * sn + zi * cs;
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
	// the lanes' partial sums of a bin count below the CTA width (complex for
	// the shifting extractor)
	return g.nbins < kThreads ? (size_t)g.nb * g.nbins * (kThreads / g.nbins) * sizeof(float) * (g.shift ? 2 : 1) : 0;
}

size_t pcal_smem(size_t group_smem, int tpc) { return (sizeof(int4) + sizeof(int32_t)) * (size_t)tpc + group_smem; }

void launch_pcal_bin(const DevPcalGroup *groups, int ngroups, int maxbins, int nchunk, int nbits, int bpt, bool shift,
                     size_t smem, const DevStation *st, const DevSubintStation *sub, const FftParam *params,
                     const uint8_t *valid, int64_t valid_stride, int T, int64_t chunk_stride, double *bins,
                     cudaStream_t stream)
{
	if(ngroups <= 0)
		return;
	const bool swar = nbits == 2 && bpt == 32 && !shift, one = bpt <= 32;
	const int tpc = (T + nchunk - 1) / nchunk;
	const int nbb = (maxbins + kThreads - 1) / kThreads;
	const dim3 grid(nbb * ((T + tpc - 1) / tpc), ngroups);
#define FXB_BIN(B, O, W, S) k_pcal_bin<B, O, W, S><<<grid, kThreads, smem, stream>>>(groups, st, sub, params, valid, \
	                                                                            valid_stride, T, tpc, chunk_stride, bins)
	if(swar) FXB_BIN(2, true, true, false);
	else if(!shift && nbits == 2 && one) FXB_BIN(2, true, false, false);
	else if(!shift && nbits == 2) FXB_BIN(2, false, false, false);
	else if(!shift && one) FXB_BIN(8, true, false, false);
	else if(!shift) FXB_BIN(8, false, false, false);
	else if(nbits == 2 && one) FXB_BIN(2, true, false, true);
	else if(nbits == 2) FXB_BIN(2, false, false, true);
	else if(one) FXB_BIN(8, true, false, true);
	else FXB_BIN(8, false, false, true);
#undef FXB_BIN
}

cudaError_t pcal_init(size_t smem)
{
	const void *k[] = {(const void *)k_pcal_bin<2, true, true, false>, (const void *)k_pcal_bin<2, true, false, false>,
	                   (const void *)k_pcal_bin<2, false, false, false>, (const void *)k_pcal_bin<8, true, false, false>,
	                   (const void *)k_pcal_bin<8, false, false, false>, (const void *)k_pcal_bin<2, true, false, true>,
	                   (const void *)k_pcal_bin<2, false, false, true>, (const void *)k_pcal_bin<8, true, false, true>,
	                   (const void *)k_pcal_bin<8, false, false, true>};
	for(const void *f : k)
	{
		const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		if(e != cudaSuccess)
			return e;
	}
	return cudaSuccess;
}

void launch_pcal_final(const DevPcalBand *bands, int nbands, int nchunk, int64_t chunk_stride, const double *bins,
                       float2 *core, cudaStream_t stream)
{
	if(nbands > 0)
		k_pcal_final<<<nbands, kThreads, 0, stream>>>(bands, nchunk, chunk_stride, bins, core);
}

}  // namespace fxb
