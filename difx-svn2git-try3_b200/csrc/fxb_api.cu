// C ABI of the FX path (include/fxb200.h): context life cycle, device memory,
// the per-subint launch sequence and result readout.

#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <tuple>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {
cudaError_t upload_lut8(cudaStream_t stream);
}

using namespace fxb;

struct Slot {
	std::vector<uint8_t *> raw;        // device staging per station
	std::vector<int64_t> rawcap;
	uint8_t *rawall = nullptr;         // device staging of a subint whose station buffers are adjacent
	int64_t rawallcap = 0;
	DevSubintStation *d_sub = nullptr;
	int32_t *d_vflags = nullptr;
	// host side of d_sub / d_vflags: pageable, the driver stages each copy
	// before cudaMemcpyAsync returns
	DevSubintStation *h_sub = nullptr;
	int32_t *h_vflags = nullptr;
	cudaEvent_t copied = nullptr, done = nullptr;
	bool used = false;
	// kernel timing of the slot's last subint: starts of prep, F stage and
	// XMAC, end of the subint (recorded on every launch, graph nodes included);
	// tpending: recorded while timing was on and not yet added to the sums
	cudaEvent_t tev[4] = {nullptr, nullptr, nullptr, nullptr};
	bool tpending = false;
	// this slot's subint kernels as one CUDA graph, valid while the
	// frame-validity array it was captured with is current
	cudaGraphExec_t gexec = nullptr;
	const uint8_t *g_valid = nullptr;
	int64_t g_stride = 0;
	int g_gen = -1;
};

// Online autotuner (fxb_autotune): over its first subints a context tries
// scheduling candidates -- F stage: FFT iterations per CTA and grid order;
// tensor-core XMAC: raw and operand ring depths -- timing every launch with
// events, and keeps the fastest per F-stage kind and XMAC group.  None of
// them changes any arithmetic, so every candidate gives identical results.
struct Tuner {
	int iter = 0, total = 0;                             // tuning while iter < total
	std::vector<std::pair<int, int>> fc;                 // F candidates: (iterations per CTA, items fastest)
	std::vector<std::vector<float>> fms;                 // [kind][candidate] fastest launch seen (ms)
	struct XCand { int nrs, nas, nb; };
	std::vector<std::vector<XCand>> xc;                  // [group] XMAC candidates: ring depths, accumulator buffers
	std::vector<std::vector<float>> xms;                 // [group][candidate]
	std::vector<cudaEvent_t> ev;                         // boundaries: kinds (nk + 1), then groups (ng + 1)
	bool done = false;
};

struct fxb_ctx {
	Job job;
	std::string err;
	int device = 0;
	cudaStream_t stream = nullptr, copy_stream = nullptr;
	// device memory comes from this pool (a server's, whose memory stays
	// mapped between jobs) or, when null, the device's default pool; every
	// allocation and free is stream-ordered, so none synchronises the device
	cudaMemPool_t pool = nullptr;
	int S = 0, T = 0, F = 0, nflagint = 0, maxband = 0, maxN = 0, maxfft = 0;
	DevStation *d_st = nullptr;
	std::vector<DevStation> h_st;
	DevBand *d_bands = nullptr;
	DevFreqPlan *d_plans = nullptr;
	std::vector<DevFreqPlan> h_plans;
	std::vector<void *> owned;          // misc device allocations
	float2 *d_twiddle = nullptr;
	FftParam *d_params = nullptr;
	float *d_pbw = nullptr;              // per-band data weights of INTERLACEDVDIF stations [S][T][nbm]
	int nbm = 0;
	float2 *d_spec = nullptr;
	float2 *d_acc = nullptr;
	float *d_bwacc = nullptr, *d_acwacc = nullptr;
	DevBWeight *d_bw = nullptr;
	DevACWeight *d_acw = nullptr;
	DevOutMap *d_om = nullptr;
	int nbw = 0, nacw = 0, nom = 0;
	DevZoomCopy *d_zoom = nullptr;       // zoom-band rows gathered after the F stage
	int nzoom = 0;
	// phase cal: binning groups, bands, and the FP64 bins of the integration
	std::vector<DevPcalGroup> h_pgroups;
	DevPcalGroup *d_pgroups = nullptr;
	DevPcalBand *d_pbands = nullptr;
	int npbands = 0;
	int pchunks = 1;                     // chunks of FFTs, each with its own slice of the bins
	struct PcalClass { int first, count, nbits, bpt, shift, maxbins; size_t smem; };
	std::vector<PcalClass> pclass;       // runs of groups of one sample layout: one launch each
	size_t psmem = 0;
	double *d_pbins = nullptr;           // [pchunks][job.pcal_bins]
	float2 *d_core = nullptr;
	uint8_t *d_valid = nullptr;          // frame validity [S][valid_stride], then the band masks
	uint32_t *d_bandok = nullptr;        // [S][valid_stride] in the same allocation
	uint8_t *d_fillok = nullptr;         // [S][valid_stride] frames without fill pattern, same allocation
	// raw INTERLACEDVDIF reads: frame-slot tables, muxed headers and status
	// words of those stations, carved per subint from one scratch block
	int nraw = 0;
	int32_t *d_mux = nullptr;
	size_t mux_cap = 0;                  // int32 words
	int64_t valid_stride = 0;
	std::vector<Slot> slots;
	int next_slot = 0;
	int last_slot = -1;              // slot of the last submitted subint
	bool timed = false;
	// per-subint kernel timing (fxb_timing_enable / fxb_timing_read)
	bool timing_on = false;
	bool graphs = true;       // replay each slot's kernels as a CUDA graph (eager launches while timing)
	bool batched = false;     // a member of an fxb_batch: subints arrive through the batch
	Tuner tune;
	int gen = 0;              // bumped whenever launch parameters change: graphs are captured again
	// work enqueued on the context's stream since a pipelined batch last
	// ordered itself after it (a read, a reset, a reallocation)
	bool dirty = false;
	double t_prep = 0, t_f = 0, t_x = 0; // per-stage sums over timed subints (ms)
	int32_t t_n = 0;
	std::vector<bool> delay_set;
	// F-stage work items (by kind) and FP32 XMAC v2 launch groups
	FGroup *d_groups = nullptr;
	std::vector<FKind> fkinds;
	// the kinds of the persistent F launches and their work list (wide units
	// first), on the host and on the device, and the launches' unit counters
	std::vector<FsMultiKind> pkinds;
	std::vector<FsMultiUnit> punits;
	int32_t punit0[kFsMultiClasses] = {}, pnunit[kFsMultiClasses] = {};
	FsMultiKind *d_pkinds = nullptr;
	FsMultiUnit *d_punits = nullptr;
	int32_t *d_pctr = nullptr;
	void *d_specn = nullptr;             // half2 (or bf16x2) spectra of the tensor-core forms, X 2^-kTcSpecExp
	void *d_tctab = nullptr;             // constant tables of the tensor-core FFT kernel
	// XMAC launch groups (subbands of equal rows and channels); the
	// tensor-core form also keeps each group's spectra in one block
	struct XGroup {
		int plan0 = 0, nf = 0;
		bool xmac = true;                         // false: spectra only (zoom-band parents), no XMAC
		int32_t *d_idx = nullptr;
		TcShape shape{};
		int64_t spec_base = 0;                    // first bf16x2 value of the group's block
		int64_t spec8_base = 0;                   // FP8 form: first e4m3x2 word of the group's block
		alignas(64) unsigned char tmap[128];     // CUtensorMap of the block (64-byte aligned)
	};
	std::vector<XGroup> xgroups;
	// tensor-core XMAC state
	bool tc = false;
	bool f8 = false;                     // FP8 form: quantise the half2 spectra to e4m3 pairs for the XMAC
	bool h16 = false;                    // spectra (and XMAC operands unless FP8) as FP16; BF16 otherwise
	uint16_t *d_spec8 = nullptr;
	int64_t spec8_elems = 0, iscale_elems = 0;
	int nsm = 0;
	int64_t specn_elems = 0;
	int32_t *d_err = nullptr;
	cudaError_t launch_err = cudaSuccess;   // first failed kernel launch of the last launch_compute
};

static std::mutex g_err_mutex;
static std::string g_create_err;

static fxb_status cuda_fail(fxb_ctx *ctx, cudaError_t e, const char *what)
{
	char buf[512];
	snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
	if(ctx)
		ctx->err = buf;
	else
	{
		std::lock_guard<std::mutex> lk(g_err_mutex);
		g_create_err = buf;
	}
	return e == cudaErrorMemoryAllocation ? FXB_ERR_NOMEM : FXB_ERR_CUDA;
}

#define CK(ctx, call)                                  \
	do {                                               \
		cudaError_t e_ = (call);                       \
		if(e_ != cudaSuccess)                          \
			return cuda_fail((ctx), e_, #call);        \
	} while(0)

static cudaError_t pool_alloc(fxb_ctx *ctx, void **p, size_t bytes, cudaStream_t s)
{
	bytes = std::max<size_t>(bytes, 1);
	return ctx->pool ? cudaMallocFromPoolAsync(p, bytes, ctx->pool, s) : cudaMallocAsync(p, bytes, s);
}

template <typename T>
static cudaError_t dalloc(fxb_ctx *ctx, T **p, size_t n)
{
	void *v = nullptr;
	cudaError_t e = pool_alloc(ctx, &v, n * sizeof(T), ctx->stream);
	if(e == cudaSuccess)
	{
		ctx->owned.push_back(v);
		*p = (T *)v;
	}
	return e;
}

// Work units of the tensor-core FFT F stage for one kind's items (FGroups at
// absolute indices first ..): pairs of subbands of one station with equal
// sideband, as [n][2] absolute FGroup indices (-1: no second subband),
// ordered (pair position, station) so that the stations of one subband
// pair are neighbours.  False if a station's sample layout does not suit the
// kernel (2-bit, 2..32 bands alike in every station of the kind, each
// subband's bands in one 4-bit field, 16-byte aligned frames of at least 128
// samples); *bpt = bits per time.
static bool tc_fft_pairs(const Job &job, const std::vector<FGroup> &items, int first, std::vector<int32_t> &pairs,
                         int *bpt)
{
	std::map<int, std::vector<int>> bystation;
	*bpt = 0;
	for(size_t i = 0; i < items.size(); i++)
	{
		const FGroup &g = items[i];
		const Job::Station &js = job.stations[g.station];
		const int fb = js.payload + js.header;
		const int b = js.nbits * js.nband;
		const int fs = js.payload * 8 / b;
		if(js.nbits != 2 || (b != 4 && b != 8 && b != 16 && b != 32 && b != 64) || (*bpt && b != *bpt) ||
		   js.payload % 16 || js.header % 16 || fb % 16 || fs < 128)
			return false;
		*bpt = b;
		if((g.band[0] & 1) || (g.nb == 2 && g.band[1] != g.band[0] + 1))
			return false;
		bystation[g.station].push_back(first + (int)i);
	}
	std::vector<std::vector<std::pair<int, int>>> per;     // [station] pairs
	for(auto &kv : bystation)
	{
		std::vector<int> &v = kv.second;
		std::stable_sort(v.begin(), v.end(), [&](int x, int y) {
			const FGroup &a = items[x - first], &b = items[y - first];
			return a.lsb != b.lsb ? a.lsb < b.lsb : a.freq < b.freq;
		});
		std::vector<std::pair<int, int>> ps;
		for(size_t i = 0; i < v.size();)
		{
			if(i + 1 < v.size() && items[v[i] - first].lsb == items[v[i + 1] - first].lsb)
			{
				ps.push_back({v[i], v[i + 1]});
				i += 2;
			}
			else
			{
				ps.push_back({v[i], -1});
				i += 1;
			}
		}
		per.push_back(ps);
	}
	size_t most = 0;
	for(const auto &ps : per)
		most = std::max(most, ps.size());
	for(size_t k = 0; k < most; k++)
		for(const auto &ps : per)
			if(k < ps.size())
			{
				pairs.push_back(ps[k].first);
				pairs.push_back(ps[k].second);
			}
	return !pairs.empty();
}

static void free_ctx(fxb_ctx *ctx)
{
	if(!ctx)
		return;
	if(ctx->stream)
		cudaStreamSynchronize(ctx->stream);
	if(ctx->copy_stream)
		cudaStreamSynchronize(ctx->copy_stream);
	// every stream is idle: the frees, ordered on the compute stream, return
	// the memory to its pool
	for(void *p : ctx->owned)
		cudaFreeAsync(p, ctx->stream);
	if(ctx->d_valid)
		cudaFreeAsync(ctx->d_valid, ctx->stream);
	if(ctx->d_mux)
		cudaFreeAsync(ctx->d_mux, ctx->stream);
	for(auto &s : ctx->slots)
	{
		for(auto *p : s.raw)
			if(p) cudaFreeAsync(p, ctx->stream);
		if(s.rawall) cudaFreeAsync(s.rawall, ctx->stream);
	}
	if(ctx->stream)
		cudaStreamSynchronize(ctx->stream);
	for(auto &s : ctx->slots)
	{
		std::free(s.h_sub);
		std::free(s.h_vflags);
		if(s.gexec) cudaGraphExecDestroy(s.gexec);
		if(s.copied) cudaEventDestroy(s.copied);
		if(s.done) cudaEventDestroy(s.done);
	}
	for(auto &s : ctx->slots)
		for(cudaEvent_t e : s.tev)
			if(e) cudaEventDestroy(e);
	for(cudaEvent_t e : ctx->tune.ev)
		if(e) cudaEventDestroy(e);
	if(ctx->stream) cudaStreamDestroy(ctx->stream);
	if(ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
	delete ctx;
}

// Phase-cal binning groups: a station's bands with tones and equal bin
// counts, as many as fit one CTA's shared memory and kPcalGroupBands.
static std::vector<DevPcalGroup> pcal_groups(const Job &job)
{
	std::vector<DevPcalGroup> out;
	for(const Job::PcalBand &p : job.pcal)
	{
		if(p.nbins <= 0)
			continue;
		DevPcalGroup *g = nullptr;
		for(DevPcalGroup &c : out)
			if(c.station == p.station && c.nbins == p.nbins && c.shift == p.shift && c.nb < kPcalGroupBands)
			{
				DevPcalGroup t = c;
				t.nb++;
				if(pcal_group_smem(t) <= kPcalSmemMax)
					g = &c;
			}
		if(!g)
		{
			out.push_back(DevPcalGroup{});
			g = &out.back();
			memset(g, 0, sizeof(*g));
			g->station = p.station;
			g->nbins = p.nbins;
			g->shift = p.shift;
			g->fs = p.fs;
		}
		g->band[g->nb] = p.band;
		g->bin_off[g->nb] = p.bin_off;
		g->nb++;
	}
	return out;
}

// Chunks of FFTs per subint for the phase-cal binning: about four CTAs per
// SM, at most one FFT per chunk, and at most 64 MB of bins.
static int pcal_chunks(const Job &job, const std::vector<DevPcalGroup> &groups)
{
	int64_t ctas = 0;                     // CTAs of one chunk: blocks of 256 bins per group
	for(const DevPcalGroup &g : groups)
		ctas += (g.nbins + 255) / 256;
	if(ctas == 0 || job.pcal_bins <= 0)
		return 1;
	int n = (int)((600 + ctas - 1) / ctas);
	n = std::min(n, std::max(job.blockspersend, 1));
	const int64_t cap = (int64_t)(64 << 20) / (8 * job.pcal_bins);
	n = (int)std::min<int64_t>(n, std::max<int64_t>(cap, 1));
	return std::max(n, 1);
}

static fxb_status setup_device(fxb_ctx *ctx)
{
	Job &job = ctx->job;
	CK(ctx, cudaGetDevice(&ctx->device));
	CK(ctx, cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->device));
	CK(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
	CK(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
	ctx->S = (int)job.stations.size();
	ctx->T = job.blockspersend;
	ctx->F = (int)job.freqs.size();
	ctx->nflagint = ctx->T / kFlagsPerInt + 1;
	ctx->delay_set.assign(ctx->S, false);

	// stations
	ctx->h_st.resize(ctx->S);
	ctx->maxband = 0;
	ctx->maxN = 0;
	for(int s = 0; s < ctx->S; s++)
	{
		const Job::Station &js = job.stations[s];
		DevStation &d = ctx->h_st[s];
		memset(&d, 0, sizeof(d));
		const fxb_freq &f = job.freqs[js.band_freq[0]];
		d.nbits = js.nbits;
		d.payload = js.payload;
		d.header = js.header;
		d.nband = js.nband;
		// a complex sample holds a real and an imaginary field (mode.cpp:51-59,
		// 77-82, 140-143; format_vdif.c:3828-3849)
		const int cpl = js.cplx ? 2 : 1;
		d.cplx = js.cplx ? 1 : 0;
		d.framebytes = js.payload + js.header;
		d.framesamples = js.payload * 8 / (js.nbits * js.nband * cpl);
		d.gran = 8 / (js.nband * js.nbits * cpl);
		if(d.gran <= 0) d.gran = 1;
		d.nchan = f.nchan;
		d.fftchannels = js.cplx ? f.nchan : 2 * f.nchan;
		d.asl = calcstridelength((unsigned)f.nchan);
		// 8-bit decoders that stop advancing in a blanked frame: real 2 and 4
		// channels (format_vdif.c:1879-1922), complex 1, 2 and 4 (:2829-2955)
		d.sticky = (js.nbits == 8 && (js.cplx ? js.nband <= 4 : (js.nband == 2 || js.nband == 4))) ? 1 : 0;
		d.mux = js.mux_threads > 0 ? 1 : 0;
		if(d.mux)
			ctx->nbm = std::max(ctx->nbm, js.nband);
		if(js.mux_raw)
		{
			d.muxraw = 1;
			d.nthr = js.mux_threads;
			d.inframebytes = js.payload / js.mux_threads + 32;
			const double fps = 2.0 * f.bw_mhz * 1e6 / d.framesamples;
			d.fps = (int)(fps + 0.5);
			if(std::fabs(fps - d.fps) > 1e-9 || d.fps < 1)
			{
				ctx->err = "raw INTERLACEDVDIF reads need a whole number of frames per second";
				return FXB_ERR_UNSUPPORTED;
			}
			for(int t = 0; t < js.mux_threads; t++)
				d.tmap[t] = js.mux_tids[t];
			ctx->nraw++;
		}
		d.bpbn = (js.nband * 1 * js.nbits * cpl) / 8;
		d.bpbd = 1;
		if(d.bpbn == 0)
		{
			d.bpbn = 1;
			d.bpbd = 8 / (js.nband * js.nbits * cpl);
		}
		d.bw = f.bw_mhz;
		d.sampletime = js.cplx ? 1.0 / f.bw_mhz : 1.0 / (2.0 * f.bw_mhz);
		ctx->maxband = std::max(ctx->maxband, js.nband);
		ctx->maxN = std::max(ctx->maxN, d.fftchannels);
	}
	ctx->maxfft = ctx->maxN;
	CK(ctx, dalloc(ctx, &ctx->d_st, ctx->S));
	CK(ctx, cudaMemcpyAsync(ctx->d_st, ctx->h_st.data(), sizeof(DevStation) * ctx->S, cudaMemcpyHostToDevice, ctx->stream));

	// bands
	std::vector<DevBand> hb((size_t)ctx->S * ctx->maxband);
	for(int s = 0; s < ctx->S; s++)
		for(int b = 0; b < ctx->maxband; b++)
		{
			DevBand &d = hb[(size_t)s * ctx->maxband + b];
			memset(&d, 0, sizeof(d));
			d.row = -1;
			if(b >= job.stations[s].nband) continue;
			int f = job.stations[s].band_freq[b];
			d.freq = f;
			d.row = job.band_row[s][b];
			d.lsb = job.freqs[f].lower_sideband;
			d.lofreq = job.freqs[f].freq_mhz;
		}
	CK(ctx, dalloc(ctx, &ctx->d_bands, hb.size()));
	CK(ctx, cudaMemcpyAsync(ctx->d_bands, hb.data(), sizeof(DevBand) * hb.size(), cudaMemcpyHostToDevice, ctx->stream));

	// twiddles exp(-2 pi i k / maxN), computed in double
	{
		std::vector<float2> tw(ctx->maxN);
		for(int k = 0; k < ctx->maxN; k++)
		{
			double ang = -2.0 * M_PI * (double)k / (double)ctx->maxN;
			tw[k] = make_float2((float)cos(ang), (float)sin(ang));
		}
		CK(ctx, dalloc(ctx, &ctx->d_twiddle, tw.size()));
		CK(ctx, cudaMemcpyAsync(ctx->d_twiddle, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice, ctx->stream));
	}

	// per-frequency plans
	ctx->h_plans.assign(ctx->F, DevFreqPlan{});
	for(int f = 0; f < ctx->F; f++)
	{
		const Job::FreqPlan &p = job.plan[f];
		DevFreqPlan &d = ctx->h_plans[f];
		memset(&d, 0, sizeof(d));
		d.nrow = p.nrow;
		d.nchan = p.nchan;
		if(p.nrow == 0) continue;
		d.ntr = (p.nrow + kTile - 1) / kTile;
		d.npair = d.ntr * (d.ntr + 1) / 2;
		d.spec_off = p.spec_off;
		d.acc_off = p.acc_off;
		d.acc_cstride = 1;
		d.acc_ostride = p.nchan;
		int32_t *dA, *dB;
		int16_t *pairs;
		CK(ctx, dalloc(ctx, &dA, p.destA.size()));
		CK(ctx, dalloc(ctx, &dB, p.destB.size()));
		CK(ctx, cudaMemcpyAsync(dA, p.destA.data(), sizeof(int32_t) * p.destA.size(), cudaMemcpyHostToDevice, ctx->stream));
		CK(ctx, cudaMemcpyAsync(dB, p.destB.data(), sizeof(int32_t) * p.destB.size(), cudaMemcpyHostToDevice, ctx->stream));
		std::vector<int16_t> hp;
		for(int i = 0; i < d.ntr; i++)
			for(int j = i; j < d.ntr; j++)
			{
				hp.push_back((int16_t)i);
				hp.push_back((int16_t)j);
			}
		CK(ctx, dalloc(ctx, &pairs, hp.size()));
		CK(ctx, cudaMemcpyAsync(pairs, hp.data(), sizeof(int16_t) * hp.size(), cudaMemcpyHostToDevice, ctx->stream));
		d.destA = dA;
		d.destB = dB;
		d.pairs = pairs;
		// inverse of destA / destB: which input pair (and whether conjugated) feeds each output
		{
			std::vector<int32_t> src((size_t)std::max(p.nout, 1), -1);
			for(int a = 0; a < p.nrow; a++)
				for(int b = a; b < p.nrow; b++)
				{
					const int oA = p.destA[(size_t)a * p.nrow + b], oB = p.destB[(size_t)a * p.nrow + b];
					if(oA >= 0 && oA < p.nout) src[oA] = a | (b << 8);
					if(oB >= 0 && oB < p.nout) src[oB] = a | (b << 8) | (1 << 16);
				}
			int32_t *ds = nullptr;
			CK(ctx, dalloc(ctx, &ds, src.size()));
			CK(ctx, cudaMemcpyAsync(ds, src.data(), sizeof(int32_t) * src.size(), cudaMemcpyHostToDevice, ctx->stream));
			d.outsrc = ds;
		}
	}
	// XMAC launch groups: frequencies with equal shape share a launch
	ctx->tc = job.xmac_kind == FXB_XMAC_BF16 || job.xmac_kind == FXB_XMAC_FP8 || job.xmac_kind == FXB_XMAC_FP16;
	ctx->f8 = job.xmac_kind == FXB_XMAC_FP8;
	ctx->h16 = job.xmac_kind == FXB_XMAC_FP16 || job.xmac_kind == FXB_XMAC_FP8;
	std::vector<std::vector<int32_t>> gidx;
	{
		std::vector<int> used;
		for(int f = 0; f < ctx->F; f++)
			if(ctx->h_plans[f].nrow > 0) used.push_back(f);
		std::vector<int> taken(used.size(), 0);
		for(size_t i = 0; i < used.size(); i++)
		{
			if(taken[i]) continue;
			const DevFreqPlan &a = ctx->h_plans[used[i]];
			std::vector<int32_t> idx;
			const bool ax = job.plan[used[i]].xmac;
			for(size_t j = i; j < used.size(); j++)
			{
				const DevFreqPlan &b = ctx->h_plans[used[j]];
				if(!taken[j] && b.nrow == a.nrow && b.nchan == a.nchan && job.plan[used[j]].xmac == ax)
				{
					taken[j] = 1;
					idx.push_back(used[j]);
				}
			}
			ctx->xgroups.emplace_back();
			ctx->xgroups.back().plan0 = used[i];
			ctx->xgroups.back().nf = (int)idx.size();
			ctx->xgroups.back().xmac = ax;
			gidx.push_back(idx);
		}
	}
	// tensor-core form: bf16x2 spectra, per group one block
	// [subband][Tpad][nrow][nchan] (times past T stay zero), and
	// [chan][output] accumulators
	if(ctx->tc)
	{
		int64_t off = 0;
		std::vector<int64_t> isoff(ctx->F, -1);   // FP8 form: each subband's first scale
		for(size_t gi = 0; gi < ctx->xgroups.size(); gi++)
		{
			fxb_ctx::XGroup &g = ctx->xgroups[gi];
			const DevFreqPlan &p0 = ctx->h_plans[g.plan0];
			if(!tc_shape(p0.nrow, p0.nchan, ctx->T, ctx->f8, ctx->h16, &g.shape))
			{
				ctx->err = "tensor-core XMAC: at most 64 inputs per subband";
				return FXB_ERR_UNSUPPORTED;
			}
			g.spec_base = off;
			g.spec8_base = ctx->spec8_elems;
			const int nblk = (p0.nchan + g.shape.CB - 1) / g.shape.CB;
			const int64_t per = (int64_t)g.shape.Tpad * nblk * p0.nrow * g.shape.CB;
			const int64_t per8 = (int64_t)g.shape.Tpad * nblk * g.shape.w8;
			for(size_t i = 0; i < gidx[gi].size(); i++)
			{
				DevFreqPlan &d = ctx->h_plans[gidx[gi][i]];
				d.spec_off = off + (int64_t)i * per;
				d.spec8_off = ctx->spec8_elems + (int64_t)i * per8;
				isoff[gidx[gi][i]] = ctx->iscale_elems;
				ctx->iscale_elems += (int64_t)d.nchan * d.nrow;
				d.tcb = g.shape.CB;
				d.tnblk = nblk;
				d.acc_ostride = 1;
				d.acc_cstride = job.plan[gidx[gi][i]].nout;
			}
			off += per * (int64_t)gidx[gi].size();
			ctx->spec8_elems += per8 * (int64_t)gidx[gi].size();
		}
		ctx->specn_elems = off;
		if(ctx->f8)
		{
			// e4m3x2 spectra (times past T stay zero) and the per-(channel, input) scales
			CK(ctx, dalloc(ctx, &ctx->d_spec8, (size_t)ctx->spec8_elems));
			CK(ctx, cudaMemsetAsync(ctx->d_spec8, 0, sizeof(uint16_t) * (size_t)ctx->spec8_elems, ctx->stream));
			float *isc = nullptr;
			CK(ctx, dalloc(ctx, &isc, (size_t)ctx->iscale_elems));
			for(int f = 0; f < ctx->F; f++)
				ctx->h_plans[f].iscale = isoff[f] >= 0 ? isc + isoff[f] : nullptr;
		}
	}
	CK(ctx, dalloc(ctx, &ctx->d_plans, ctx->F));
	CK(ctx, cudaMemcpyAsync(ctx->d_plans, ctx->h_plans.data(), sizeof(DevFreqPlan) * ctx->F, cudaMemcpyHostToDevice, ctx->stream));
	for(size_t gi = 0; gi < ctx->xgroups.size(); gi++)
	{
		fxb_ctx::XGroup &g = ctx->xgroups[gi];
		CK(ctx, dalloc(ctx, &g.d_idx, gidx[gi].size()));
		CK(ctx, cudaMemcpyAsync(g.d_idx, gidx[gi].data(), sizeof(int32_t) * gidx[gi].size(), cudaMemcpyHostToDevice, ctx->stream));
	}
	if(ctx->tc)
	{
		uint32_t *sn = nullptr;
		CK(ctx, dalloc(ctx, &sn, (size_t)ctx->specn_elems));
		CK(ctx, cudaMemsetAsync(sn, 0, sizeof(uint32_t) * (size_t)ctx->specn_elems, ctx->stream));
		ctx->d_specn = sn;
		CK(ctx, dalloc(ctx, &ctx->d_err, 1));
		CK(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(int32_t), ctx->stream));
		CK(ctx, cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->device));
		for(fxb_ctx::XGroup &g : ctx->xgroups)
			if(tc_tensormap_size() > sizeof(g.tmap) ||
			   !tc_make_tensormap(g.tmap, ctx->f8 ? (const void *)(ctx->d_spec8 + g.spec8_base) : (const void *)(sn + g.spec_base),
			                      g.shape, g.nf))
			{
				ctx->err = "cuTensorMapEncodeTiled failed for the spectra buffer";
				return FXB_ERR_CUDA;
			}
	}

	// F-stage work items: (station, subband) with up to two bands each, one
	// launch per kind (FFT length, bands per item)
	{
		const int out = ctx->tc ? 1 : 0;
		std::map<std::pair<int, int>, std::vector<FGroup>> bykind;
		for(int s = 0; s < ctx->S; s++)
		{
			const Job::Station &js = job.stations[s];
			const int N = ctx->h_st[s].fftchannels;
			const bool pairs = N <= 2048;
			std::vector<int> done(js.nband, 0);
			for(int b = 0; b < js.nband; b++)
			{
				if(done[b] || job.band_row[s][b] < 0)
					continue;
				const int f = js.band_freq[b];
				int b1 = -1;
				if(pairs)
					for(int c = b + 1; c < js.nband; c++)
						if(!done[c] && js.band_freq[c] == f && job.band_row[s][c] >= 0)
						{
							b1 = c;
							break;
						}
				done[b] = 1;
				if(b1 >= 0) done[b1] = 1;
				FGroup g;
				memset(&g, 0, sizeof(g));
				g.station = s;
				g.freq = f;
				g.band[0] = b;
				g.band[1] = b1 >= 0 ? b1 : b;
				g.row[0] = job.band_row[s][b];
				g.row[1] = b1 >= 0 ? job.band_row[s][b1] : -1;
				g.nb = b1 >= 0 ? 2 : 1;
				g.lsb = job.freqs[f].lower_sideband;
				g.lofreq = job.freqs[f].freq_mhz;
				// complex lower sideband: the effective LO is at negative
				// frequency (mode.cpp:899-903)
				if(js.cplx && g.lsb)
					g.lofreq = -g.lofreq;
				if(js.has_corr)
				{
					// the phase offset rotates the non-R band of the frequency's
					// first two bands, or the first when neither is R
					// (mode.cpp:1336-1347)
					int q0 = -1, q1 = -1;
					for(int c = 0; c < js.nband && q1 < 0; c++)
						if(js.band_freq[c] == f)
						{
							if(q0 < 0)
								q0 = c;
							else
								q1 = c;
						}
					const int lcp = q1 < 0 ? -1 : (js.band_pol[q0] == 'R' ? q1 : q0);
					for(int j = 0; j < 2; j++)
					{
						const int bj = g.band[j];
						g.clk[j] = js.clk[bj] - (js.band_pol[bj] == 'R' ? 0.5 : -0.5) * js.dclk[bj];
						g.phase[j] = bj == lcp ? (float)(js.phase[bj] / 720.0) : 0.0f;
					}
					g.looff = js.looff[b];
					g.corr = 1;
				}
				// raw INTERLACEDVDIF reads and complex sampling take their own
				// kernel instantiations
				bykind[{N, g.nb + (ctx->h_st[s].muxraw ? 16 : 0) + (ctx->h_st[s].cplx ? 32 : 0)}].push_back(g);
			}
		}
		std::vector<FGroup> hg;
		if(out == 1)
		{
			// all stations of a subband side by side in the grid: their rows of
			// one spectra block are written close together in time
			for(auto &kv : bykind)
				std::stable_sort(kv.second.begin(), kv.second.end(),
				                 [](const FGroup &x, const FGroup &y) { return x.freq < y.freq; });
		}
		for(const auto &kv : bykind)
		{
			FKind k;
			memset(&k, 0, sizeof(k));
			if(!fstage_plan(kv.first.first, kv.first.second & 15, out, &k))
			{
				ctx->err = "F stage: no kernel shape for FFT length " + std::to_string(kv.first.first);
				return FXB_ERR_UNSUPPORTED;
			}
			k.muxraw = (kv.first.second >> 4) & 1;
			k.cplx = (kv.first.second >> 5) & 1;
			k.first = (int)hg.size();
			k.count = (int)kv.second.size();
			// FFT iterations per CTA: as many as still leave two CTAs per SM
			for(int tq : {4, 2, 1})
			{
				k.tq = tq;
				const int per = tq * k.fpc;
				if((int64_t)((ctx->T + per - 1) / per) * k.count >= 2 * (int64_t)ctx->nsm)
					break;
			}
			// tensor-core form at N = 2048: the FFT runs on the tensor cores
			// (fxb_fstage_tc.cu) wherever the stations' sample layout allows it
			// (FXB_TC_FFT=0 selects the CUDA-core FP16 F stage instead)
			if(out == 1)
			{
				bool any_lsb = false;
				for(const FGroup &gg : kv.second)
					any_lsb = any_lsb || gg.lsb;
				const char *env = getenv("FXB_TC_FFT");
				// no EDV4 band blanking and no complex sampling there
				const bool allow = !(env && env[0] == '0') && ctx->nbm == 0 && !k.cplx;
				std::vector<int32_t> pairs;
				int bpt = 0;
				if(allow && fstage_tc_eligible(k.N, job.fringe_rot_order, any_lsb) &&
				   tc_fft_pairs(job, kv.second, (int)hg.size(), pairs, &bpt))
				{
					if(!ctx->d_tctab)
					{
						std::vector<unsigned char> h(fstage_tc_tables_bytes());
						make_fstage_tc_tables(h.data());
						unsigned char *d = nullptr;
						CK(ctx, dalloc(ctx, &d, h.size()));
						CK(ctx, cudaMemcpyAsync(d, h.data(), h.size(), cudaMemcpyHostToDevice, ctx->stream));
						ctx->d_tctab = d;
					}
					int32_t *dp = nullptr;
					CK(ctx, dalloc(ctx, &dp, pairs.size()));
					CK(ctx, cudaMemcpyAsync(dp, pairs.data(), sizeof(int32_t) * pairs.size(), cudaMemcpyHostToDevice,
					                        ctx->stream));
					k.tcfft = 1;
					k.tctab = ctx->d_tctab;
					k.tcpairs = dp;
					k.tcnpairs = (int32_t)(pairs.size() / 2);
					k.tcbpt = bpt;
				}
			}
			{
				std::vector<float2> h((size_t)k.twn);
				make_fstage_twiddles(k.N, h.data());
				float2 *d = nullptr;
				CK(ctx, dalloc(ctx, &d, h.size()));
				CK(ctx, cudaMemcpyAsync(d, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice, ctx->stream));
				k.tw = d;
			}
			bool wide = false;
			if(out == 1 && !k.tcfft && !k.cplx && fstage_multi_shape(k.N, k.nb, &wide))
				k.persist = 1;
			hg.insert(hg.end(), kv.second.begin(), kv.second.end());
			ctx->fkinds.push_back(k);
		}
		// the persistent launches' work list: per kind tq x fpc FFT times of
		// one item per unit, times outer and items inner
		{
			// classes: wide, two-band narrow, one-band narrow units of plain
			// VDIF, then of raw reads
			std::vector<FsMultiUnit> cls[kFsMultiClasses];
			for(const FKind &k : ctx->fkinds)
			{
				if(!k.persist)
					continue;
				bool w = false;
				fstage_multi_shape(k.N, k.nb, &w);
				FsMultiKind mk;
				memset(&mk, 0, sizeof(mk));
				mk.tw = k.tw;
				int logn = 0;
				while((1 << logn) < k.N)
					logn++;
				mk.code = 128 * k.muxraw + 32 * k.nb + logn;
				mk.first = k.first;
				mk.tq = fstage_multi_tq(k.N, k.nb, k.tq);
				const int ki = (int)ctx->pkinds.size();
				ctx->pkinds.push_back(mk);
				const int per = mk.tq * k.fpc, nt = (ctx->T + per - 1) / per;
				std::vector<FsMultiUnit> &dst = cls[3 * k.muxraw + (w ? 0 : 3 - k.nb)];
				for(int t = 0; t < nt; t++)
					for(int it = 0; it < k.count; it++)
						dst.push_back(FsMultiUnit{ki, it, t});
			}
			for(int c = 0; c < kFsMultiClasses; c++)
			{
				ctx->punit0[c] = (int32_t)ctx->punits.size();
				ctx->pnunit[c] = (int32_t)cls[c].size();
				ctx->punits.insert(ctx->punits.end(), cls[c].begin(), cls[c].end());
			}
			if(!ctx->pkinds.empty())
			{
				CK(ctx, dalloc(ctx, &ctx->d_pkinds, ctx->pkinds.size()));
				CK(ctx, dalloc(ctx, &ctx->d_punits, ctx->punits.size()));
				CK(ctx, dalloc(ctx, &ctx->d_pctr, kFsMultiClasses));
				CK(ctx, cudaMemcpyAsync(ctx->d_pkinds, ctx->pkinds.data(), sizeof(FsMultiKind) * ctx->pkinds.size(),
				                        cudaMemcpyHostToDevice, ctx->stream));
				CK(ctx, cudaMemcpyAsync(ctx->d_punits, ctx->punits.data(), sizeof(FsMultiUnit) * ctx->punits.size(),
				                        cudaMemcpyHostToDevice, ctx->stream));
			}
		}
		CK(ctx, dalloc(ctx, &ctx->d_groups, std::max<size_t>(hg.size(), 1)));
		if(!hg.empty())
			CK(ctx, cudaMemcpyAsync(ctx->d_groups, hg.data(), sizeof(FGroup) * hg.size(), cudaMemcpyHostToDevice, ctx->stream));
	}
	// big buffers
	CK(ctx, dalloc(ctx, &ctx->d_params, (size_t)ctx->S * ctx->T));
	if(ctx->nbm)
		CK(ctx, dalloc(ctx, &ctx->d_pbw, (size_t)ctx->S * ctx->T * ctx->nbm));
	CK(ctx, dalloc(ctx, &ctx->d_spec, job.xmac_kind == FXB_XMAC_FP32 ? (size_t)job.spec_total : 1));
	CK(ctx, dalloc(ctx, &ctx->d_acc, (size_t)job.acc_total));
	CK(ctx, dalloc(ctx, &ctx->d_core, (size_t)job.corelen));
	ctx->nbw = (int)job.bweights.size();
	ctx->nacw = (int)job.acweights.size();
	ctx->nom = (int)job.outmap.size();
	CK(ctx, dalloc(ctx, &ctx->d_bwacc, ctx->nbw));
	CK(ctx, dalloc(ctx, &ctx->d_acwacc, ctx->nacw));
	{
		std::vector<DevBWeight> hbw(ctx->nbw);
		for(int i = 0; i < ctx->nbw; i++)
			hbw[i] = DevBWeight{job.bweights[i].s1, job.bweights[i].s2, job.bweights[i].b1, job.bweights[i].b2,
			                    job.bweights[i].dst_float};
		std::vector<DevACWeight> hacw(ctx->nacw);
		for(int i = 0; i < ctx->nacw; i++)
			hacw[i] = DevACWeight{job.acweights[i].s, job.acweights[i].band, job.acweights[i].dst_float};
		std::vector<DevOutMap> hom(ctx->nom);
		for(int i = 0; i < ctx->nom; i++)
		{
			const Job::OutMap &m = job.outmap[i];
			int64_t a = m.acc;
			int cs = 1;
			if(ctx->tc && m.out >= 0)
			{
				a = job.plan[m.freq].acc_off + m.out;
				cs = job.plan[m.freq].nout;
			}
			hom[i] = DevOutMap{a, m.core, m.nchan, m.avg, cs, 0};
		}
		CK(ctx, dalloc(ctx, &ctx->d_bw, ctx->nbw));
		CK(ctx, dalloc(ctx, &ctx->d_acw, ctx->nacw));
		CK(ctx, dalloc(ctx, &ctx->d_om, ctx->nom));
		if(ctx->nbw) CK(ctx, cudaMemcpyAsync(ctx->d_bw, hbw.data(), sizeof(DevBWeight) * ctx->nbw, cudaMemcpyHostToDevice, ctx->stream));
		if(ctx->nacw) CK(ctx, cudaMemcpyAsync(ctx->d_acw, hacw.data(), sizeof(DevACWeight) * ctx->nacw, cudaMemcpyHostToDevice, ctx->stream));
		if(ctx->nom) CK(ctx, cudaMemcpyAsync(ctx->d_om, hom.data(), sizeof(DevOutMap) * ctx->nom, cudaMemcpyHostToDevice, ctx->stream));
		// phase cal: binning groups, every band's tones for the DFT, and one
		// slice of FP64 bins per chunk of FFTs
		{
			std::vector<DevPcalBand> hb;
			for(const Job::PcalBand &p : job.pcal)
				hb.push_back(DevPcalBand{p.ntones, p.nbins, p.first, p.step, p.shift, 0, p.bin_off, p.core});
			ctx->h_pgroups = pcal_groups(job);
			auto class_of = [&](const DevPcalGroup &g) {
				const Job::Station &js = job.stations[g.station];
				return std::make_tuple(js.nbits, js.nbits * js.nband, g.shift != 0);
			};
			std::stable_sort(ctx->h_pgroups.begin(), ctx->h_pgroups.end(),
			                 [&](const DevPcalGroup &x, const DevPcalGroup &y) { return class_of(x) < class_of(y); });
			ctx->pchunks = pcal_chunks(job, ctx->h_pgroups);
			// chunks of a multiple of four FFTs, so that the 2 or 4 lanes of a
			// bin (bin counts of 128 or 64) share a chunk evenly
			int tpc = (ctx->T + ctx->pchunks - 1) / ctx->pchunks;
			tpc = std::min(ctx->T, (tpc + 3) / 4 * 4);
			// and short enough that the chunk's FFT table and the lane sums fit
			// one CTA's shared memory
			size_t lanes = 0;
			for(const DevPcalGroup &g : ctx->h_pgroups)
				lanes = std::max(lanes, pcal_group_smem(g));
			while(tpc > 4 && pcal_smem(lanes, tpc) > kPcalSmemLaunchMax)
				tpc = (tpc / 2 + 3) / 4 * 4;
			ctx->pchunks = (ctx->T + tpc - 1) / tpc;
			for(size_t i = 0; i < ctx->h_pgroups.size(); i++)
			{
				const DevPcalGroup &g = ctx->h_pgroups[i];
				const auto c = class_of(g);
				if(ctx->pclass.empty() || ctx->pclass.back().nbits != std::get<0>(c) ||
				   ctx->pclass.back().bpt != std::get<1>(c) || ctx->pclass.back().shift != (int)std::get<2>(c))
					ctx->pclass.push_back({(int)i, 0, std::get<0>(c), std::get<1>(c), (int)std::get<2>(c), 0, 0});
				fxb_ctx::PcalClass &pc = ctx->pclass.back();
				pc.count++;
				pc.maxbins = std::max(pc.maxbins, g.nbins);
				pc.smem = std::max(pc.smem, pcal_smem(pcal_group_smem(g), tpc));
				ctx->psmem = std::max(ctx->psmem, pc.smem);
			}
			ctx->npbands = (int)hb.size();
			if(ctx->npbands)
			{
				if(ctx->psmem)
					CK(ctx, pcal_init(ctx->psmem));
				CK(ctx, dalloc(ctx, &ctx->d_pbands, hb.size()));
				CK(ctx, cudaMemcpyAsync(ctx->d_pbands, hb.data(), sizeof(DevPcalBand) * hb.size(), cudaMemcpyHostToDevice, ctx->stream));
				CK(ctx, dalloc(ctx, &ctx->d_pgroups, std::max<size_t>(ctx->h_pgroups.size(), 1)));
				if(!ctx->h_pgroups.empty())
					CK(ctx, cudaMemcpyAsync(ctx->d_pgroups, ctx->h_pgroups.data(), sizeof(DevPcalGroup) * ctx->h_pgroups.size(),
					                        cudaMemcpyHostToDevice, ctx->stream));
				const size_t nbins = (size_t)ctx->pchunks * (size_t)std::max<int64_t>(job.pcal_bins, 1);
				CK(ctx, dalloc(ctx, &ctx->d_pbins, nbins));
				CK(ctx, cudaMemsetAsync(ctx->d_pbins, 0, sizeof(double) * nbins, ctx->stream));
			}
		}
		ctx->nzoom = (int)job.zooms.size();
		if(ctx->nzoom)
		{
			std::vector<DevZoomCopy> hz(ctx->nzoom);
			for(int i = 0; i < ctx->nzoom; i++)
			{
				const Job::ZoomCopy &z = job.zooms[i];
				hz[i] = DevZoomCopy{z.src_freq, z.src_row, z.dst_freq, z.dst_row, z.choff, z.nchan};
			}
			CK(ctx, dalloc(ctx, &ctx->d_zoom, ctx->nzoom));
			CK(ctx, cudaMemcpyAsync(ctx->d_zoom, hz.data(), sizeof(DevZoomCopy) * ctx->nzoom, cudaMemcpyHostToDevice, ctx->stream));
		}
	}

	// staging slots
	ctx->slots.resize(job.inflight);
	for(auto &sl : ctx->slots)
	{
		sl.raw.assign(ctx->S, nullptr);
		sl.rawcap.assign(ctx->S, 0);
		CK(ctx, dalloc(ctx, &sl.d_sub, ctx->S));
		CK(ctx, dalloc(ctx, &sl.d_vflags, (size_t)ctx->S * ctx->nflagint));
		sl.h_sub = (DevSubintStation *)std::calloc(ctx->S, sizeof(DevSubintStation));
		sl.h_vflags = (int32_t *)std::calloc((size_t)ctx->S * ctx->nflagint, sizeof(int32_t));
		if(!sl.h_sub || !sl.h_vflags)
		{
			ctx->err = "host allocation failed";
			return FXB_ERR_NOMEM;
		}
		CK(ctx, cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming));
		CK(ctx, cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
		for(cudaEvent_t &e : sl.tev)
			CK(ctx, cudaEventCreate(&e));
	}
	CK(ctx, upload_lut8(ctx->stream));
	CK(ctx, cudaMemsetAsync(ctx->d_acc, 0, sizeof(float2) * std::max<int64_t>(job.acc_total, 1), ctx->stream));
	CK(ctx, cudaMemsetAsync(ctx->d_bwacc, 0, sizeof(float) * std::max(ctx->nbw, 1), ctx->stream));
	CK(ctx, cudaMemsetAsync(ctx->d_acwacc, 0, sizeof(float) * std::max(ctx->nacw, 1), ctx->stream));
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	return FXB_OK;
}

namespace fxb {

fxb_ctx *create_ctx(const fxb_job_desc *desc, void *pool, fxb_status *status)
{
	fxb_ctx *ctx = new fxb_ctx;
	ctx->pool = (cudaMemPool_t)pool;
	fxb_status st = FXB_OK;
	std::string err;
	if(!build_job(desc, ctx->job, err, st))
	{
		{
			std::lock_guard<std::mutex> lk(g_err_mutex);
			g_create_err = err;
		}
		delete ctx;
		if(status) *status = st;
		return nullptr;
	}
	st = setup_device(ctx);
	if(st != FXB_OK)
	{
		{
			std::lock_guard<std::mutex> lk(g_err_mutex);
			g_create_err = ctx->err;
		}
		free_ctx(ctx);
		if(status) *status = st;
		return nullptr;
	}
	if(status) *status = FXB_OK;
	return ctx;
}

bool ctx_slot_free(fxb_ctx *ctx)
{
	const auto &sl = ctx->slots[ctx->next_slot];
	return !sl.used || cudaEventQuery(sl.done) != cudaErrorNotReady;
}

}  // namespace fxb

extern "C" {

fxb_ctx *fxb_create(const fxb_job_desc *desc, fxb_status *status) { return fxb::create_ctx(desc, nullptr, status); }

void fxb_destroy(fxb_ctx *ctx) { free_ctx(ctx); }

const char *fxb_last_error(const fxb_ctx *ctx)
{
	if(ctx)
		return ctx->err.c_str();
	std::lock_guard<std::mutex> lk(g_err_mutex);
	return g_create_err.c_str();
}

fxb_status fxb_set_delay_poly(fxb_ctx *ctx, int32_t station, int32_t npoly, int32_t order, double poly0_sec,
                              int32_t interval_s, const double *coeffs)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx) return FXB_ERR_ARG;
	if(station < 0 || station >= ctx->S || npoly < 1 || npoly > kMaxPolys || order < 0 || order > kMaxPolyOrder ||
	   interval_s <= 0 || !coeffs)
	{
		ctx->err = "bad delay polynomial";
		return FXB_ERR_ARG;
	}
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	DevStation &d = ctx->h_st[station];
	d.npoly = npoly;
	d.order = order;
	d.interval = interval_s;
	d.poly0 = poly0_sec;
	memset(d.coeffs, 0, sizeof(d.coeffs));
	memcpy(d.coeffs, coeffs, sizeof(double) * npoly * (order + 1));
	CK(ctx, cudaMemcpyAsync(ctx->d_st + station, &d, sizeof(DevStation), cudaMemcpyHostToDevice, ctx->stream));
	ctx->delay_set[station] = true;
	return FXB_OK;
}

// Adds a completed slot's kernel times to the context's sums (timing on).
static void slot_account(fxb_ctx *ctx, Slot &sl)
{
	if(!sl.tpending)
		return;
	sl.tpending = false;
	float a = 0, b = 0, c = 0;
	if(cudaEventElapsedTime(&a, sl.tev[0], sl.tev[1]) == cudaSuccess &&
	   cudaEventElapsedTime(&b, sl.tev[1], sl.tev[2]) == cudaSuccess &&
	   cudaEventElapsedTime(&c, sl.tev[2], sl.tev[3]) == cudaSuccess)
	{
		ctx->t_prep += a;
		ctx->t_f += b;
		ctx->t_x += c;
		ctx->t_n++;
	}
	else
		cudaGetLastError();
}

// Waits for the next slot, fills its per-station records and queues the
// copies of this subint's station buffers on the copy stream; the slot's
// `copied` event marks their end.
static fxb_status stage_subint(fxb_ctx *ctx, const uint8_t *const *bufs, const int64_t *nbytes,
                               const int32_t *datasec, const int32_t *datans, const int32_t *const *validflags,
                               int32_t sec, int32_t ns, bool device, Slot **slot, const double *interp = nullptr)
{
	if(!ctx || !bufs || !nbytes || !datasec || !datans)
		return FXB_ERR_ARG;
	for(int s = 0; s < ctx->S && !interp; s++)
		if(!ctx->delay_set[s])
		{
			ctx->err = "delay model not set for every station";
			return FXB_ERR_STATE;
		}
	const Job &job = ctx->job;
	Slot &sl = ctx->slots[ctx->next_slot];
	ctx->next_slot = (ctx->next_slot + 1) % (int)ctx->slots.size();
	if(sl.used)
		CK(ctx, cudaEventSynchronize(sl.done));
	slot_account(ctx, sl);
	sl.used = true;

	// frame-validity array sized for the largest buffer of this subint
	int64_t need = 0;
	for(int s = 0; s < ctx->S; s++)
	{
		if(nbytes[s] < 0 || (nbytes[s] > 0 && !bufs[s]))
		{
			ctx->err = "bad station buffer";
			return FXB_ERR_ARG;
		}
		need = std::max<int64_t>(need, nbytes[s] / ctx->h_st[s].payload + 2);
	}
	if(need > ctx->valid_stride)
	{
		// stream-ordered: the earlier subints' kernels finish with the old array first
		if(ctx->d_valid)
		{
			CK(ctx, cudaFreeAsync(ctx->d_valid, ctx->stream));
		ctx->dirty = true;
			ctx->d_valid = nullptr;
		}
		const size_t vbytes = ((size_t)need * ctx->S + 15) / 16 * 16;
		CK(ctx, pool_alloc(ctx, (void **)&ctx->d_valid, 2 * vbytes + sizeof(uint32_t) * need * ctx->S, ctx->stream));
		ctx->d_bandok = (uint32_t *)(ctx->d_valid + vbytes);
		ctx->d_fillok = ctx->d_valid + vbytes + sizeof(uint32_t) * need * ctx->S;
		ctx->valid_stride = need;
	}

	// raw INTERLACEDVDIF reads: slot tables, muxed headers and status words
	// (shared by the staging slots: their kernels run in stream order)
	std::vector<size_t> mux_off(ctx->S, 0);
	if(ctx->nraw)
	{
		size_t words = 0;
		for(int s = 0; s < ctx->S; s++)
		{
			const DevStation &d = ctx->h_st[s];
			if(!d.muxraw)
				continue;
			const int64_t nin = nbytes[s] / d.inframebytes;
			mux_off[s] = words;
			words += (size_t)(4 * nin / d.nthr) * d.nthr + (size_t)(nin / d.nthr + 1) * 16 + 4;
			words = (words + 3) & ~(size_t)3;
		}
		if(words > ctx->mux_cap)
		{
			if(ctx->d_mux)
				CK(ctx, cudaFreeAsync(ctx->d_mux, ctx->stream));
			ctx->dirty = true;
			ctx->d_mux = nullptr;
			CK(ctx, pool_alloc(ctx, (void **)&ctx->d_mux, sizeof(int32_t) * words, ctx->stream));
			ctx->mux_cap = words;
		}
	}

	// host buffers one after the other (as a datastream's receive ring holds
	// them) with 16-byte aligned starts: one copy for the whole subint
	bool merged = !device && ctx->S > 1;
	int64_t total = 0;
	for(int s = 0; s < ctx->S && merged; s++)
	{
		if(bufs[s] != bufs[0] + total || (total & 15) != 0)
			merged = false;
		total += nbytes[s];
	}
	if(merged && total > 0)
	{
		if(sl.rawallcap < total)
		{
			if(sl.rawall) CK(ctx, cudaFreeAsync(sl.rawall, ctx->copy_stream));
			sl.rawall = nullptr;
			const int64_t cap = total + total / 8 + 4096;
			CK(ctx, pool_alloc(ctx, (void **)&sl.rawall, cap, ctx->copy_stream));
			sl.rawallcap = cap;
		}
		CK(ctx, cudaMemcpyAsync(sl.rawall, bufs[0], total, cudaMemcpyHostToDevice, ctx->copy_stream));
	}
	int64_t off = 0;
	for(int s = 0; s < ctx->S; s++)
	{
		DevSubintStation &u = sl.h_sub[s];
		memset(&u, 0, sizeof(u));
		u.nbytes = nbytes[s];
		u.datasec = datasec[s];
		u.datans = datans[s];
		u.subsec = sec;
		u.subns = ns;
		if(ctx->h_st[s].muxraw)
		{
			const DevStation &d = ctx->h_st[s];
			u.mux_nin = (int32_t)(nbytes[s] / d.inframebytes);
			u.mux_nproc = u.mux_nin / d.nthr;
			u.mux_nslot = 4 * u.mux_nin / d.nthr;
			u.mux_slot = ctx->d_mux + mux_off[s];
			u.mux_hdr = (uint32_t *)(u.mux_slot + (size_t)u.mux_nslot * d.nthr);
			u.mux_status = (int32_t *)(u.mux_hdr + (size_t)(u.mux_nproc + 1) * 16);
		}
		if(interp)
		{
			// the caller's interpolator (Mode::setOffsets' own, mode.cpp:1541-1554);
			// NaN: no model for this time, the subint is torched
			u.interp_given = 1;
			u.interp[0] = interp[3 * s];
			u.interp[1] = interp[3 * s + 1];
			u.interp[2] = interp[3 * s + 2];
			u.invalid_subint = std::isnan(interp[3 * s]) ? 1 : 0;
		}
		if(device)
			u.buf = bufs[s];
		else if(merged)
		{
			u.buf = sl.rawall + off;
			off += nbytes[s];
		}
		else
		{
			if(sl.rawcap[s] < nbytes[s])
			{
				// the slot is idle (its done event has completed), so the old
				// buffer can go back at once; the new one is ordered on the
				// copy stream ahead of the copy into it
				if(sl.raw[s]) CK(ctx, cudaFreeAsync(sl.raw[s], ctx->copy_stream));
				sl.raw[s] = nullptr;
				int64_t cap = nbytes[s] + nbytes[s] / 8 + 4096;
				CK(ctx, pool_alloc(ctx, (void **)&sl.raw[s], cap, ctx->copy_stream));
				sl.rawcap[s] = cap;
			}
			u.buf = sl.raw[s];
			if(nbytes[s] > 0)
				CK(ctx, cudaMemcpyAsync(sl.raw[s], bufs[s], nbytes[s], cudaMemcpyHostToDevice, ctx->copy_stream));
		}
		int32_t *vf = sl.h_vflags + (size_t)s * ctx->nflagint;
		if(validflags && validflags[s])
			memcpy(vf, validflags[s], sizeof(int32_t) * ((ctx->T + kFlagsPerInt - 1) / kFlagsPerInt));
		else
			for(int k = 0; k < ctx->nflagint; k++) vf[k] = 0x3FFFFFFF;
	}
	CK(ctx, cudaMemcpyAsync(sl.d_sub, sl.h_sub, sizeof(DevSubintStation) * ctx->S, cudaMemcpyHostToDevice, ctx->copy_stream));
	CK(ctx, cudaMemcpyAsync(sl.d_vflags, sl.h_vflags, sizeof(int32_t) * ctx->S * ctx->nflagint, cudaMemcpyHostToDevice,
	                        ctx->copy_stream));
	CK(ctx, cudaEventRecord(sl.copied, ctx->copy_stream));
	*slot = &sl;
	return FXB_OK;
}

// Every kernel of one subint whose inputs sit in slot sl, on stream st.  No
// host synchronisation and no argument that changes between subints (the
// subint time travels in the slot's records), so that the sequence can be
// captured once per slot and replayed.  capture: the slot's four timing
// events become event-record nodes of the graph.
// Delay interpolators, raw-read placement, frame validity and per-FFT
// parameters of one subint (Mode::setOffsets, Mk5Mode::unpack's checks).
static void launch_prep(fxb_ctx *ctx, const Slot &sl, cudaStream_t st, unsigned evf)
{
	const Job &job = ctx->job;
	cudaEventRecordWithFlags(sl.tev[0], st, evf);
	if(ctx->nraw)
	{
		launch_interpolators(ctx->d_st, sl.d_sub, ctx->S, ctx->T, st);
		launch_mux_raw(ctx->d_st, sl.d_sub, ctx->S, 0, 0, st);
		launch_frame_valid(ctx->d_st, sl.d_sub, ctx->d_valid, ctx->d_bandok, ctx->valid_stride, ctx->S, st,
		                   ctx->d_fillok);
	}
	else
		fxb::launch_prep(ctx->d_st, sl.d_sub, ctx->S, ctx->T, ctx->d_valid, ctx->d_bandok, ctx->valid_stride, st,
		                 ctx->d_fillok);
	launch_fft_params(ctx->d_st, sl.d_sub, sl.d_vflags, ctx->nflagint, ctx->d_valid, ctx->d_bandok, ctx->valid_stride,
	                  ctx->S, ctx->T, job.fringe_rot_order, ctx->d_params, ctx->d_pbw, ctx->nbm, st, ctx->d_fillok);
	cudaEventRecordWithFlags(sl.tev[1], st, evf);
}

// The F-stage arguments of one subint (every kind but the twiddles and the
// scheduling fields).
static FsArgs fs_args(const fxb_ctx *ctx, const Slot &sl)
{
	const Job &job = ctx->job;
	FsArgs fa;
	memset(&fa, 0, sizeof(fa));
	fa.st = ctx->d_st;
	fa.sub = sl.d_sub;
	fa.groups = ctx->d_groups;
	fa.plans = ctx->d_plans;
	fa.valid = ctx->d_valid;
	fa.bandok = ctx->nbm ? ctx->d_bandok : nullptr;
	fa.fillok = ctx->d_fillok;
	fa.valid_stride = ctx->valid_stride;
	fa.params = ctx->d_params;
	fa.maxN = ctx->maxN;
	fa.T = ctx->T;
	fa.order = job.fringe_rot_order;
	fa.fraclo = job.fractionallofreq ? 1 : 0;
	fa.spec = ctx->tc ? ctx->d_specn : (void *)ctx->d_spec;
	fa.err = ctx->d_err;
	fa.h16 = ctx->h16 ? 1 : 0;
	return fa;
}

static void launch_xmac_weights(fxb_ctx *ctx, const Slot &sl, cudaStream_t st, unsigned evf, bool tuning,
                                bool xmac = true);

static void launch_compute(fxb_ctx *ctx, const Slot &sl, cudaStream_t st, bool capture)
{
	Tuner &tn = ctx->tune;
	const bool tuning = !capture && tn.iter < tn.total;
	const size_t nk = ctx->fkinds.size();
	const unsigned evf = capture ? cudaEventRecordExternal : cudaEventRecordDefault;
	launch_prep(ctx, sl, st, evf);
	{
		const FsArgs fa = fs_args(ctx, sl);
		for(size_t i = 0; i < nk; i++)
		{
			FKind k = ctx->fkinds[i];
			if(tuning)
				cudaEventRecord(tn.ev[i], st);
			if(k.persist)
				continue;
			if(tuning)
			{
				if(!k.tcfft)
				{
					const auto &c = tn.fc[tn.iter % tn.fc.size()];
					k.tq = c.first;
					k.items_fast = c.second;
				}
			}
			if(k.tcfft)
			{
				const cudaError_t le = launch_fstage_tc(k, fa, ctx->nsm, st);
				if(le != cudaSuccess && ctx->launch_err == cudaSuccess)
					ctx->launch_err = le;
			}
			else
				launch_fstage_kind(k, fa, st);
		}
		if(!ctx->pkinds.empty())
		{
			FsMultiArgs ma;
			memset(&ma, 0, sizeof(ma));
			ma.m[0] = fa;
			ma.kinds = ctx->d_pkinds;
			ma.units = ctx->d_punits;
			for(int c = 0; c < kFsMultiClasses; c++)
			{
				ma.unit0[c] = ctx->punit0[c];
				ma.nunit[c] = ctx->pnunit[c];
			}
			ma.ctr = ctx->d_pctr;
			cudaMemsetAsync(ctx->d_pctr, 0, kFsMultiClasses * sizeof(int32_t), st);
			const cudaError_t le = launch_fstage_multi(ma, ctx->nsm, st);
			if(le != cudaSuccess && ctx->launch_err == cudaSuccess)
				ctx->launch_err = le;
		}
		if(tuning)
			cudaEventRecord(tn.ev[nk], st);
	}
	launch_xmac_weights(ctx, sl, st, evf, tuning);
}

// Phase-cal bins and zoom gathers (after the F stage), the FP8 quantisation,
// every XMAC group (unless xmac is false: the caller runs them) and the
// weights of one subint.
static void launch_xmac_weights(fxb_ctx *ctx, const Slot &sl, cudaStream_t st, unsigned evf, bool tuning, bool xmac)
{
	const Job &job = ctx->job;
	Tuner &tn = ctx->tune;
	const size_t nk = ctx->fkinds.size();
	for(const auto &pc : ctx->pclass)
		launch_pcal_bin(ctx->d_pgroups + pc.first, pc.count, pc.maxbins, ctx->pchunks, pc.nbits, pc.bpt, pc.shift != 0,
		                pc.smem, ctx->d_st, sl.d_sub, ctx->d_params, ctx->d_valid, ctx->valid_stride, ctx->T,
		                job.pcal_bins, ctx->d_pbins, st);
	launch_zoom_gather(ctx->d_zoom, ctx->nzoom, ctx->d_plans, ctx->T, ctx->tc,
	                   ctx->tc ? ctx->d_specn : (void *)ctx->d_spec, st);
	cudaEventRecordWithFlags(sl.tev[2], st, evf);
	if(ctx->f8)
		for(const auto &g : ctx->xgroups)
			if(g.xmac)
				launch_quant_fp8(g.shape, ctx->d_plans, g.d_idx, g.nf, ctx->T, (const uint32_t *)ctx->d_specn,
				                 ctx->d_spec8, st);
	for(size_t gi = 0; gi < ctx->xgroups.size(); gi++)
	{
		const auto &g = ctx->xgroups[gi];
		TcShape sh = g.shape;
		if(tuning)
			cudaEventRecord(tn.ev[nk + 1 + gi], st);
		if(!g.xmac || !xmac)
			continue;
		if(tuning)
		{
			if(ctx->tc && !tn.xc[gi].empty())
			{
				const auto &c = tn.xc[gi][tn.iter % tn.xc[gi].size()];
				tc_stages(&sh, c.nrs, c.nas, c.nb);
			}
		}
		if(ctx->tc)
			launch_xmac_tc(g.tmap, sh, ctx->d_plans, g.d_idx, g.nf, ctx->nsm, ctx->d_err, ctx->d_acc, st);
		else
			launch_xmac_fp32v2(ctx->h_plans[g.plan0], ctx->d_plans, g.d_idx, g.nf, ctx->T, ctx->d_spec, ctx->d_acc, st);
	}
	if(tuning)
		cudaEventRecord(tn.ev[nk + 1 + ctx->xgroups.size()], st);
	launch_weights(ctx->d_bw, ctx->nbw, ctx->d_acw, ctx->nacw, ctx->d_params, ctx->d_pbw, ctx->nbm, ctx->d_st, ctx->T,
	               ctx->d_bwacc, ctx->d_acwacc, st);
	cudaEventRecordWithFlags(sl.tev[3], st, evf);
	// a launch that could not start (resources, configuration) leaves its
	// error behind; keep it for the submit to report
	const cudaError_t le = cudaPeekAtLastError();
	if(le != cudaSuccess && ctx->launch_err == cudaSuccess)
		ctx->launch_err = le;
}

// The first kernel-launch failure recorded by launch_compute since the last
// call, as a status (cleared).
static fxb_status take_launch_err(fxb_ctx *ctx)
{
	const cudaError_t e = ctx->launch_err;
	if(e == cudaSuccess)
		return FXB_OK;
	ctx->launch_err = cudaSuccess;
	cudaGetLastError();
	ctx->err = std::string("kernel launch failed: ") + cudaGetErrorString(e);
	return FXB_ERR_CUDA;
}

// Reads one tuning subint's launch times (waits for it), and after the last
// one keeps each kind's and group's fastest candidate.
static void tune_collect(fxb_ctx *ctx)
{
	Tuner &t = ctx->tune;
	const size_t nk = ctx->fkinds.size(), ng = ctx->xgroups.size();
	if(cudaEventSynchronize(t.ev.back()) == cudaSuccess)
	{
		float ms = 0;
		for(size_t i = 0; i < nk; i++)
			if(cudaEventElapsedTime(&ms, t.ev[i], t.ev[i + 1]) == cudaSuccess)
			{
				float &best = t.fms[i][t.iter % t.fc.size()];
				best = std::min(best, ms);
			}
		for(size_t g = 0; g < ng; g++)
			if(!t.xc[g].empty() && cudaEventElapsedTime(&ms, t.ev[nk + 1 + g], t.ev[nk + 2 + g]) == cudaSuccess)
			{
				float &best = t.xms[g][t.iter % t.xc[g].size()];
				best = std::min(best, ms);
			}
	}
	cudaGetLastError();
	if(++t.iter < t.total)
		return;
	for(size_t i = 0; i < nk; i++)
	{
		if(ctx->fkinds[i].tcfft || ctx->fkinds[i].persist)
			continue;
		const size_t c = std::min_element(t.fms[i].begin(), t.fms[i].end()) - t.fms[i].begin();
		ctx->fkinds[i].tq = t.fc[c].first;
		ctx->fkinds[i].items_fast = t.fc[c].second;
	}
	for(size_t g = 0; g < ng; g++)
	{
		if(t.xc[g].empty())
			continue;
		const size_t c = std::min_element(t.xms[g].begin(), t.xms[g].end()) - t.xms[g].begin();
		tc_stages(&ctx->xgroups[g].shape, t.xc[g][c].nrs, t.xc[g][c].nas, t.xc[g][c].nb);
	}
	t.done = true;
	ctx->gen++;
}

// The slot's graph, captured (again) when missing or when the frame-validity
// array has been reallocated since.  A capture that fails turns graphs off
// for the context and leaves the stream as it was.
static fxb_status slot_graph(fxb_ctx *ctx, Slot &sl)
{
	if(sl.gexec && sl.g_valid == ctx->d_valid && sl.g_stride == ctx->valid_stride && sl.g_gen == ctx->gen)
		return FXB_OK;
	if(sl.gexec)
	{
		cudaGraphExecDestroy(sl.gexec);
		sl.gexec = nullptr;
	}
	CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
	launch_compute(ctx, sl, ctx->stream, true);
	cudaGraph_t g = nullptr;
	cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
	if(e == cudaSuccess)
		e = cudaGraphInstantiate(&sl.gexec, g, 0);
	if(g)
		cudaGraphDestroy(g);
	if(e != cudaSuccess)
	{
		cudaGetLastError();
		sl.gexec = nullptr;
		ctx->graphs = false;
		return FXB_OK;
	}
	sl.g_valid = ctx->d_valid;
	sl.g_stride = ctx->valid_stride;
	sl.g_gen = ctx->gen;
	return FXB_OK;
}

static fxb_status submit(fxb_ctx *ctx, const uint8_t *const *bufs, const int64_t *nbytes, const int32_t *datasec,
                         const int32_t *datans, const int32_t *const *validflags, int32_t sec, int32_t ns, bool device,
                         const double *interp = nullptr)
{
	if(ctx && ctx->batched)
	{
		ctx->err = "context belongs to a batch: submit through fxb_batch_submit";
		return FXB_ERR_STATE;
	}
	Slot *slp = nullptr;
	const fxb_status rc = stage_subint(ctx, bufs, nbytes, datasec, datans, validflags, sec, ns, device, &slp, interp);
	if(rc != FXB_OK)
		return rc;
	Slot &sl = *slp;
	cudaStream_t st = ctx->stream;
	CK(ctx, cudaStreamWaitEvent(st, sl.copied, 0));
	const bool tuning = ctx->tune.iter < ctx->tune.total;
	if(ctx->graphs && !tuning)
	{
		const fxb_status gs = slot_graph(ctx, sl);
		if(gs != FXB_OK)
			return gs;
	}
	if(ctx->graphs && !tuning)
		CK(ctx, cudaGraphLaunch(sl.gexec, st));
	else
		launch_compute(ctx, sl, st, false);
	{
		const fxb_status le = take_launch_err(ctx);
		if(le != FXB_OK)
			return le;
	}
	if(tuning)
		tune_collect(ctx);
	CK(ctx, cudaGetLastError());
	CK(ctx, cudaEventRecord(sl.done, st));
	sl.tpending = ctx->timing_on;
	ctx->last_slot = (int)(slp - ctx->slots.data());
	ctx->timed = true;
	return FXB_OK;
}

fxb_status fxb_set_graphs(fxb_ctx *ctx, int32_t on)
{
	if(!ctx) return FXB_ERR_ARG;
	ctx->graphs = on != 0;
	return FXB_OK;
}

fxb_status fxb_autotune(fxb_ctx *ctx, int32_t rounds)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx || rounds < 0)
		return FXB_ERR_ARG;
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	Tuner &t = ctx->tune;
	for(cudaEvent_t e : t.ev)
		if(e) cudaEventDestroy(e);
	t = Tuner();
	if(rounds == 0)
		return FXB_OK;
	const size_t nk = ctx->fkinds.size(), ng = ctx->xgroups.size();
	t.fc = {{4, 1}, {4, 0}, {2, 1}, {2, 0}, {1, 1}, {1, 0}};
	t.fms.assign(nk, std::vector<float>(t.fc.size(), 1e30f));
	t.xc.assign(ng, {});
	size_t most = t.fc.size();
	for(size_t g = 0; g < ng && ctx->tc; g++)
	{
		if(!ctx->xgroups[g].xmac)
			continue;
		// one CTA per SM with double-buffered accumulators, or two per SM
		static const int depth[][3] = {{6, 4, 2}, {6, 3, 2}, {4, 3, 2}, {4, 2, 2}, {3, 2, 2}, {2, 2, 2},
		                               {4, 2, 1}, {3, 2, 1}, {2, 2, 1}};
		for(const auto &d : depth)
		{
			TcShape sh = ctx->xgroups[g].shape;
			if(tc_stages(&sh, d[0], d[1], d[2]))
				t.xc[g].push_back({d[0], d[1], d[2]});
		}
		most = std::max(most, t.xc[g].size());
	}
	t.xms.assign(ng, std::vector<float>(most, 1e30f));
	t.ev.assign(nk + ng + 2, nullptr);
	for(cudaEvent_t &e : t.ev)
		CK(ctx, cudaEventCreate(&e));
	t.total = rounds * (int)most;
	return FXB_OK;
}

fxb_status fxb_tuning_report(const fxb_ctx *ctx, char *buf, size_t len, size_t *needed)
{
	if(!ctx)
		return FXB_ERR_ARG;
	const Tuner &t = ctx->tune;
	std::string r;
	char line[256];
	for(size_t i = 0; i < ctx->fkinds.size(); i++)
	{
		const FKind &k = ctx->fkinds[i];
		if(k.persist)
			snprintf(line, sizeof(line), "fstage N=%d items=%d: persistent launch, %d FFT iterations per unit", k.N,
			         k.count, fstage_multi_tq(k.N, k.nb, k.tq));
		else
			snprintf(line, sizeof(line), "fstage N=%d items=%d%s: %d FFT iterations per CTA, %s fastest", k.N, k.count,
			         k.tcfft ? " tensor-core FFT" : "", k.tq, k.items_fast ? "items" : "times");
		r += line;
		if(t.done && !k.tcfft && !k.persist)
			for(size_t c = 0; c < t.fc.size(); c++)
			{
				snprintf(line, sizeof(line), "%s(%d,%s) %.4f ms", c ? ", " : " | ", t.fc[c].first,
				         t.fc[c].second ? "items" : "times", (double)t.fms[i][c]);
				r += line;
			}
		r += "\n";
	}
	for(size_t g = 0; g < ctx->xgroups.size(); g++)
	{
		const TcShape &sh = ctx->xgroups[g].shape;
		if(!ctx->xgroups[g].xmac)
		{
			snprintf(line, sizeof(line), "xmac group %zu (%d inputs, %d channels): spectra only (zoom-band parents)\n",
			         g, sh.nrow, sh.nchan);
			r += line;
			continue;
		}
		if(!ctx->tc)
		{
			snprintf(line, sizeof(line), "xmac group %zu: FP32 form\n", g);
			r += line;
			continue;
		}
		snprintf(line, sizeof(line), "xmac group %zu (%d inputs, %d channels): rings %d raw / %d operand, %d CTA(s) per SM",
		         g, sh.nrow, sh.nchan, sh.nrs, sh.nas, sh.nb == 1 ? 2 : 1);
		r += line;
		if(t.done)
			for(size_t c = 0; c < t.xc[g].size(); c++)
			{
				snprintf(line, sizeof(line), "%s(%d,%d,%s) %.4f ms", c ? ", " : " | ", t.xc[g][c].nrs, t.xc[g][c].nas,
				         t.xc[g][c].nb == 1 ? "2/SM" : "1/SM", (double)t.xms[g][c]);
				r += line;
			}
		r += "\n";
	}
	if(needed)
		*needed = r.size() + 1;
	if(buf && len)
	{
		const size_t n = std::min(len - 1, r.size());
		memcpy(buf, r.data(), n);
		buf[n] = 0;
	}
	return FXB_OK;
}

fxb_status fxb_submit_subint(fxb_ctx *ctx, const uint8_t *const *bufs, const int64_t *nbytes, const int32_t *datasec,
                             const int32_t *datans, const int32_t *const *validflags, int32_t sec, int32_t ns)
{
	return submit(ctx, bufs, nbytes, datasec, datans, validflags, sec, ns, false);
}

fxb_status fxb_submit_subint_interp(fxb_ctx *ctx, const uint8_t *const *bufs, const int64_t *nbytes,
                                    const int32_t *datasec, const int32_t *datans, const int32_t *const *validflags,
                                    int32_t sec, int32_t ns, const double *interp)
{
	if(!interp)
		return FXB_ERR_ARG;
	return submit(ctx, bufs, nbytes, datasec, datans, validflags, sec, ns, false, interp);
}

fxb_status fxb_submit_subint_device(fxb_ctx *ctx, const uint8_t *const *dev_bufs, const int64_t *nbytes,
                                    const int32_t *datasec, const int32_t *datans, const int32_t *const *validflags,
                                    int32_t sec, int32_t ns)
{
	return submit(ctx, dev_bufs, nbytes, datasec, datans, validflags, sec, ns, true);
}

static fxb_status check_device_error(fxb_ctx *ctx)
{
	if(!ctx->d_err)
		return FXB_OK;
	int32_t e = 0;
	CK(ctx, cudaMemcpy(&e, ctx->d_err, sizeof(e), cudaMemcpyDeviceToHost));
	if(e)
	{
		ctx->err = "a bounded device wait expired in the tensor-core XMAC (code " + std::to_string(e) + ")";
		return FXB_ERR_TIMEOUT;
	}
	return FXB_OK;
}

fxb_status fxb_sync(fxb_ctx *ctx)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx) return FXB_ERR_ARG;
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	CK(ctx, cudaStreamSynchronize(ctx->copy_stream));
	return check_device_error(ctx);
}

fxb_status fxb_core_result_length(const fxb_ctx *ctx, int64_t *ncomplex)
{
	if(!ctx || !ncomplex) return FXB_ERR_ARG;
	*ncomplex = ctx->job.corelen;
	return FXB_OK;
}

// The layout offsets; the phase-cal offsets too when out has room for them.
static fxb_status write_layout(const Job &j, int32_t *out, size_t nint)
{
	const size_t need = 2 * j.bloff.size() + 2 * j.acoff.size();
	if(nint < need) return FXB_ERR_ARG;
	size_t k = 0;
	for(auto v : j.bloff) out[k++] = (int32_t)v;
	for(auto v : j.bwoff) out[k++] = (int32_t)v;
	for(auto v : j.acoff) out[k++] = (int32_t)v;
	for(auto v : j.acwoff) out[k++] = (int32_t)v;
	if(nint >= need + j.pcoff.size())
		for(auto v : j.pcoff) out[k++] = (int32_t)v;
	return FXB_OK;
}

fxb_status fxb_layout(const fxb_ctx *ctx, int32_t *out, size_t nint)
{
	if(!ctx || !out) return FXB_ERR_ARG;
	return write_layout(ctx->job, out, nint);
}

fxb_status fxb_job_layout(const fxb_job_desc *desc, int32_t *out, size_t nint, int64_t *ncomplex)
{
	Job job;
	std::string err;
	fxb_status st = FXB_OK;
	if(!build_job(desc, job, err, st))
	{
		std::lock_guard<std::mutex> lk(g_err_mutex);
		g_create_err = err;
		return st;
	}
	if(out)
	{
		const fxb_status ls = write_layout(job, out, nint);
		if(ls != FXB_OK) return ls;
	}
	if(ncomplex) *ncomplex = job.corelen;
	return FXB_OK;
}

fxb_status fxb_job_footprint(const fxb_job_desc *desc, size_t *bytes)
{
	if(!desc || !bytes)
		return FXB_ERR_ARG;
	Job job;
	std::string err;
	fxb_status st = FXB_OK;
	if(!build_job(desc, job, err, st))
	{
		std::lock_guard<std::mutex> lk(g_err_mutex);
		g_create_err = err;
		return st;
	}
	const int64_t T = job.blockspersend;
	const int S = (int)job.stations.size();
	// spectra (the blocked tensor-core layout pads times to 32 -- 64 for the
	// e4m3 copy of the FP8 form -- and channels to whole blocks: at most
	// +25 %), accumulators, core result, FFT parameters
	const double pad32 = (double)((T + 31) / 32 * 32) / (double)std::max<int64_t>(T, 1);
	const double pad64 = (double)((T + 63) / 64 * 64) / (double)std::max<int64_t>(T, 1);
	double b = (double)job.spec_total * (job.xmac_kind == FXB_XMAC_FP32 ? 8.0
	                                     : job.xmac_kind != FXB_XMAC_FP8 ? 4.0 * 1.25 * pad32
	                                                                      : (4.0 * pad64 + 2.0 * pad64 + 0.5) * 1.25);
	b += (double)job.acc_total * 8.0 + (double)job.corelen * 16.0 + (double)S * T * 64.0 +
	     (double)job.pcal_bins * 8.0 * pcal_chunks(job, pcal_groups(job));
	// raw VDIF staging of the in-flight subints (payload plus headers, 1/8 slack)
	for(int s = 0; s < S; s++)
	{
		const Job::Station &js = job.stations[s];
		const fxb_freq &f = job.freqs[js.band_freq[0]];
		const double sps = 2.0 * f.bw_mhz * 1e6;
		const double per = (double)job.subint_ns * 1e-9 * sps * js.nbits * js.nband / 8.0 *
		                   (double)(js.payload + js.header) / js.payload;
		b += job.inflight * (per * 1.125 + 2.0 * (js.payload + js.header) + 4096.0);
	}
	b += 16.0 * 1024 * 1024;           // plans, tables, validity bytes, alignment
	*bytes = (size_t)b;
	return FXB_OK;
}

fxb_status fxb_read_results(fxb_ctx *ctx, float *coreresult, size_t nfloats)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx || !coreresult) return FXB_ERR_ARG;
	if(nfloats < (size_t)(2 * ctx->job.corelen))
	{
		ctx->err = "result buffer too small";
		return FXB_ERR_ARG;
	}
	launch_finalise(ctx->d_om, ctx->nom, 0, ctx->d_acc, ctx->d_bw, ctx->nbw, ctx->d_bwacc, ctx->d_acw, ctx->nacw,
	                ctx->d_acwacc, ctx->d_core, ctx->job.corelen, ctx->stream);
	launch_pcal_final(ctx->d_pbands, ctx->npbands, ctx->pchunks, ctx->job.pcal_bins, ctx->d_pbins, ctx->d_core, ctx->stream);
	CK(ctx, cudaGetLastError());
	CK(ctx, cudaMemcpyAsync(coreresult, ctx->d_core, sizeof(float2) * ctx->job.corelen, cudaMemcpyDeviceToHost, ctx->stream));
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	return check_device_error(ctx);
}

fxb_status fxb_reset(fxb_ctx *ctx)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx) return FXB_ERR_ARG;
	CK(ctx, cudaMemsetAsync(ctx->d_acc, 0, sizeof(float2) * std::max<int64_t>(ctx->job.acc_total, 1), ctx->stream));
	CK(ctx, cudaMemsetAsync(ctx->d_bwacc, 0, sizeof(float) * std::max(ctx->nbw, 1), ctx->stream));
	CK(ctx, cudaMemsetAsync(ctx->d_acwacc, 0, sizeof(float) * std::max(ctx->nacw, 1), ctx->stream));
	if(ctx->d_pbins)
		CK(ctx, cudaMemsetAsync(ctx->d_pbins, 0,
		                        sizeof(double) * (size_t)ctx->pchunks * (size_t)std::max<int64_t>(ctx->job.pcal_bins, 1),
		                        ctx->stream));
	return FXB_OK;
}

fxb_status fxb_last_timing(const fxb_ctx *ctx, float *fstage_ms, float *xmac_ms, float *total_ms)
{
	if(!ctx || !ctx->timed || ctx->last_slot < 0) return FXB_ERR_STATE;
	fxb_ctx *c = const_cast<fxb_ctx *>(ctx);
	const Slot &sl = ctx->slots[ctx->last_slot];
	CK(c, cudaEventSynchronize(sl.tev[3]));
	float a = 0, b = 0, t = 0;
	CK(c, cudaEventElapsedTime(&a, sl.tev[1], sl.tev[2]));
	CK(c, cudaEventElapsedTime(&b, sl.tev[2], sl.tev[3]));
	CK(c, cudaEventElapsedTime(&t, sl.tev[0], sl.tev[3]));
	if(fstage_ms) *fstage_ms = a;
	if(xmac_ms) *xmac_ms = b;
	if(total_ms) *total_ms = t;
	return FXB_OK;
}

fxb_status fxb_timing_enable(fxb_ctx *ctx, int32_t on)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx) return FXB_ERR_ARG;
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	for(Slot &sl : ctx->slots)
		sl.tpending = false;
	ctx->timing_on = on != 0;
	ctx->t_prep = ctx->t_f = ctx->t_x = 0;
	ctx->t_n = 0;
	return FXB_OK;
}

fxb_status fxb_timing_read(fxb_ctx *ctx, int32_t *nsubint, double *prep_ms, double *fstage_ms, double *xmac_ms)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx) return FXB_ERR_ARG;
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	for(Slot &sl : ctx->slots)
		slot_account(ctx, sl);
	if(nsubint) *nsubint = ctx->t_n;
	if(prep_ms) *prep_ms = ctx->t_prep;
	if(fstage_ms) *fstage_ms = ctx->t_f;
	if(xmac_ms) *xmac_ms = ctx->t_x;
	ctx->t_prep = ctx->t_f = ctx->t_x = 0;
	ctx->t_n = 0;
	return FXB_OK;
}

fxb_status fxb_get_stream(const fxb_ctx *ctx, void **stream)
{
	if(!ctx || !stream) return FXB_ERR_ARG;
	*stream = (void *)ctx->stream;
	return FXB_OK;
}

fxb_status fxb_vdif_mux(const uint8_t *dev_in, int64_t inbytes, int32_t nthreads, const int32_t *thread_ids,
                        int32_t inframebytes, int32_t frames_per_second, int32_t nbits, uint8_t *dev_out,
                        int64_t outcap, int64_t *outbytes, void *stream)
{
	std::string err;
	const fxb_status st = vdif_mux(dev_in, inbytes, nthreads, thread_ids, inframebytes, frames_per_second, nbits,
	                               dev_out, outcap, outbytes, stream, err);
	if(st != FXB_OK)
	{
		std::lock_guard<std::mutex> lk(g_err_mutex);
		g_create_err = err.empty() ? "fxb_vdif_mux: bad arguments or CUDA error" : err;
	}
	return st;
}

static fxb_status job_of(const fxb_job_desc *desc, Job &job)
{
	if(!desc) return FXB_ERR_ARG;
	std::string err;
	fxb_status st = FXB_OK;
	if(!build_job(desc, job, err, st))
	{
		std::lock_guard<std::mutex> lk(g_err_mutex);
		g_create_err = err;
		return st;
	}
	return FXB_OK;
}

fxb_status fxb_vis_calibrate(const fxb_job_desc *desc, const fxb_vis_params *params, float *coreresult)
{
	Job job;
	const fxb_status st = job_of(desc, job);
	return st != FXB_OK ? st : vis_calibrate(job, params, coreresult);
}

fxb_status fxb_vis_write_pcal(const fxb_job_desc *desc, const fxb_vis_params *params, const float *coreresult,
                              const char *dir)
{
	Job job;
	fxb_status st = job_of(desc, job);
	if(st != FXB_OK)
		return st;
	std::string err;
	st = vis_pcal_write(job, params, coreresult, dir, err);
	if(st != FXB_OK)
	{
		std::lock_guard<std::mutex> lk(g_err_mutex);
		g_create_err = err;
	}
	return st;
}

fxb_status fxb_vis_write_swin(const fxb_job_desc *desc, const fxb_vis_params *params, const float *coreresult,
                              const char *dir)
{
	Job job;
	fxb_status st = job_of(desc, job);
	if(st != FXB_OK)
		return st;
	std::string err;
	st = vis_swin_write(job, params, coreresult, dir, err);
	if(st != FXB_OK)
	{
		std::lock_guard<std::mutex> lk(g_err_mutex);
		g_create_err = err;
	}
	return st;
}

void *fxb_host_alloc(size_t bytes, fxb_status *status)
{
	void *p = nullptr;
	const cudaError_t e = cudaHostAlloc(&p, std::max<size_t>(bytes, 1), cudaHostAllocPortable);
	if(status) *status = e == cudaSuccess ? FXB_OK : e == cudaErrorMemoryAllocation ? FXB_ERR_NOMEM : FXB_ERR_CUDA;
	return e == cudaSuccess ? p : nullptr;
}

void fxb_host_free(void *p)
{
	if(p)
		cudaFreeHost(p);
}

fxb_status fxb_read_results_device(fxb_ctx *ctx, float *dev_out, size_t nfloats)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx || !dev_out) return FXB_ERR_ARG;
	if(nfloats < (size_t)(2 * ctx->job.corelen))
	{
		ctx->err = "result buffer too small";
		return FXB_ERR_ARG;
	}
	launch_finalise(ctx->d_om, ctx->nom, 0, ctx->d_acc, ctx->d_bw, ctx->nbw, ctx->d_bwacc, ctx->d_acw, ctx->nacw,
	                ctx->d_acwacc, (float2 *)dev_out, ctx->job.corelen, ctx->stream);
	launch_pcal_final(ctx->d_pbands, ctx->npbands, ctx->pchunks, ctx->job.pcal_bins, ctx->d_pbins, (float2 *)dev_out,
	                  ctx->stream);
	CK(ctx, cudaGetLastError());
	return FXB_OK;
}

fxb_status fxb_datastream_control(fxb_ctx *ctx, int32_t station, fxb_ring *ring, int32_t scan, int32_t sec,
                                  int32_t ns, const double *delay_us, int64_t *offset, int32_t *nbytes,
                                  int32_t *datasec, int32_t *datans, int32_t *validflags, size_t nflagint)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx || station < 0 || station >= ctx->S)
		return FXB_ERR_ARG;
	if(!delay_us && !ctx->delay_set[station])
	{
		ctx->err = "no delay model for the station";
		return FXB_ERR_STATE;
	}
	return datastream_control(ctx->job, ctx->h_st[station], station, ring, scan, sec, ns, delay_us, offset, nbytes,
	                          datasec, datans, validflags, nflagint, ctx->err);
}

fxb_status fxb_job_datastream_control(const fxb_job_desc *desc, int32_t station, int32_t npoly, int32_t order,
                                      double poly0_sec, int32_t interval_s, const double *coeffs, fxb_ring *ring,
                                      int32_t scan, int32_t sec, int32_t ns, const double *delay_us, int64_t *offset,
                                      int32_t *nbytes, int32_t *datasec, int32_t *datans, int32_t *validflags,
                                      size_t nflagint)
{
	Job job;
	std::string err;
	fxb_status st = FXB_OK;
	auto fail = [&](fxb_status code) {
		std::lock_guard<std::mutex> lk(g_err_mutex);
		g_create_err = err;
		return code;
	};
	if(!build_job(desc, job, err, st))
		return fail(st);
	if(station < 0 || station >= (int)job.stations.size() || npoly < 1 || npoly > kMaxPolys || order < 0 ||
	   order > kMaxPolyOrder || interval_s <= 0 || !coeffs)
	{
		err = "bad station or delay polynomial";
		return fail(FXB_ERR_ARG);
	}
	DevStation d;
	memset(&d, 0, sizeof(d));
	d.npoly = npoly;
	d.order = order;
	d.interval = interval_s;
	d.poly0 = poly0_sec;
	memcpy(d.coeffs, coeffs, sizeof(double) * npoly * (order + 1));
	st = datastream_control(job, d, station, ring, scan, sec, ns, delay_us, offset, nbytes, datasec, datans,
	                        validflags, nflagint, err);
	return st == FXB_OK ? st : fail(st);
}

fxb_status fxb_read_spectra(fxb_ctx *ctx, int32_t freq, float *out, size_t nfloats, int32_t *nfft, int32_t *nrow)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx || !out || freq < 0 || freq >= ctx->F) return FXB_ERR_ARG;
	const DevFreqPlan &p = ctx->h_plans[freq];
	size_t n = (size_t)ctx->T * p.nrow * p.nchan;
	if(nfloats < 2 * n) return FXB_ERR_ARG;
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	if(n && ctx->tc)
	{
		// half2 or bf16x2 [t][block][row][tcb], scaled by 2^-kTcSpecExp -> FP32 [t][row][chan]
		const size_t nb = (size_t)ctx->T * p.tnblk * p.nrow * p.tcb;
		std::vector<uint32_t> h(nb);
		CK(ctx, cudaMemcpy(h.data(), (const uint32_t *)ctx->d_specn + p.spec_off, nb * 4, cudaMemcpyDeviceToHost));
		const float unscale = (float)(1 << kTcSpecExp);
		const bool h16 = ctx->h16;
		auto bf = [h16, unscale](uint32_t v) {
			float f;
			if(h16)
			{
				__half_raw r;
				r.x = (unsigned short)v;
				f = __half2float(__half(r));
			}
			else
			{
				const uint32_t u = v << 16;
				memcpy(&f, &u, 4);
			}
			return f * unscale;
		};
		for(int t = 0; t < ctx->T; t++)
			for(int r = 0; r < p.nrow; r++)
				for(int c = 0; c < p.nchan; c++)
				{
					const uint32_t v = h[(((size_t)t * p.tnblk + c / p.tcb) * p.nrow + r) * p.tcb + c % p.tcb];
					const size_t o = ((size_t)t * p.nrow + r) * p.nchan + c;
					out[2 * o] = bf(v & 0xFFFFu);
					out[2 * o + 1] = bf(v >> 16);
				}
	}
	else if(n)
		CK(ctx, cudaMemcpy(out, ctx->d_spec + p.spec_off, sizeof(float2) * n, cudaMemcpyDeviceToHost));
	if(nfft) *nfft = ctx->T;
	if(nrow) *nrow = p.nrow;
	return FXB_OK;
}

fxb_status fxb_read_fft_weights(fxb_ctx *ctx, float *out, size_t nfloats)
{
	if(ctx)
		ctx->dirty = true;
	if(!ctx || !out) return FXB_ERR_ARG;
	size_t n = (size_t)ctx->S * ctx->T;
	if(nfloats < n) return FXB_ERR_ARG;
	CK(ctx, cudaStreamSynchronize(ctx->stream));
	std::vector<FftParam> hp(n);
	CK(ctx, cudaMemcpy(hp.data(), ctx->d_params, sizeof(FftParam) * n, cudaMemcpyDeviceToHost));
	for(size_t i = 0; i < n; i++)
		out[i] = hp[i].status == kFftOk ? hp[i].weight : 0.0f;
	return FXB_OK;
}

fxb_status fxb_vdif_unpack(const uint8_t *data, int64_t nbytes, int32_t payload, int32_t header, int32_t nchan,
                           int32_t nbits, int64_t offsetsamples, int32_t nsamp, float *out, int32_t *good)
{
	if(!data || !out || !good || nbytes <= 0 || nsamp <= 0 || offsetsamples < 0 || payload <= 0 || payload % 8 ||
	   (nbits != 2 && nbits != 8) || nchan < 1 || (nchan & (nchan - 1)) || header < 0)
		return FXB_ERR_ARG;
	if((int64_t)payload * 8 % (nchan * nbits))
		return FXB_ERR_ARG;
	const int64_t fs = (int64_t)payload * 8 / (nchan * nbits);
	const int64_t nf = (offsetsamples + nsamp - 1) / fs - offsetsamples / fs + 1;
	if(nf > 40000)
		return FXB_ERR_UNSUPPORTED;
	uint8_t *d_data = nullptr;
	float *d_out = nullptr;
	int *d_good = nullptr;
	cudaStream_t st = 0;
	fxb_status rc = FXB_OK;
	// the 8-bit table is per device: uploaded for the current one on every call
	if(upload_lut8(st) != cudaSuccess)
		return FXB_ERR_CUDA;
	if(cudaMalloc(&d_data, nbytes) != cudaSuccess || cudaMalloc(&d_out, sizeof(float) * nchan * (size_t)nsamp) != cudaSuccess ||
	   cudaMalloc(&d_good, sizeof(int)) != cudaSuccess)
		rc = FXB_ERR_NOMEM;
	if(rc == FXB_OK && cudaMemcpy(d_data, data, nbytes, cudaMemcpyHostToDevice) != cudaSuccess)
		rc = FXB_ERR_CUDA;
	if(rc == FXB_OK)
	{
		launch_vdif_unpack(d_data, nbytes, payload, header, nchan, nbits, offsetsamples, nsamp, d_out, d_good, st);
		if(cudaGetLastError() != cudaSuccess ||
		   cudaMemcpy(out, d_out, sizeof(float) * nchan * (size_t)nsamp, cudaMemcpyDeviceToHost) != cudaSuccess ||
		   cudaMemcpy(good, d_good, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
			rc = FXB_ERR_CUDA;
	}
	if(d_data) cudaFree(d_data);
	if(d_out) cudaFree(d_out);
	if(d_good) cudaFree(d_good);
	return rc;
}

// ---------------------------------------------------------------- batches
// Several contexts (e.g. one per subband shape: width, channels, bits) whose
// subints are submitted together.  Per subint every member stages its copies
// on its own copy stream; then ONE graph launch on the batch stream runs all
// members' kernels, each member a parallel branch of the graph (captured once
// per slot, replayed after).  Members stay ordinary contexts for reading and
// resetting results; their streams are ordered after every batch launch.
struct fxb_batch {
	std::vector<fxb_ctx *> m;
	cudaStream_t stream = nullptr;
	cudaEvent_t fork = nullptr, done = nullptr;
	std::vector<cudaEvent_t> join;                    // [member]
	std::vector<cudaGraphExec_t> gexec;               // [slot]
	std::vector<std::vector<const uint8_t *>> g_valid; // [slot][member] validity arrays captured with
	std::vector<std::vector<int64_t>> g_stride;
	std::vector<std::vector<int>> g_gen;
	std::vector<int> g_fused;                         // [slot] the graph runs the fused launches
	bool graphs = true;
	// fused mode: the persistent F launches' work list over all members and
	// their two unit counters
	bool fused = false;
	// fused mode pipelines subints: the XMAC of a subint runs on xstream
	// beside the next subint's F stage, so every slot has its own spectra of
	// every member (slot 0: the member's own buffer) and tensor maps over them
	std::vector<std::vector<void *>> fspec;                    // [slot][member]
	std::vector<std::vector<std::vector<TmapBytes>>> ftmap;    // [slot][member][XMAC group]
	cudaStream_t xstream = nullptr;
	std::vector<cudaEvent_t> fdone, xdone;                     // [slot]
	FsMultiKind *d_kinds = nullptr;
	FsMultiUnit *d_units = nullptr;
	int32_t unit0[kFsMultiClasses] = {}, nunit[kFsMultiClasses] = {};
	int32_t *d_ctr = nullptr;
	std::string err;
};

static void free_batch(fxb_batch *b)
{
	if(b->stream)
		cudaStreamSynchronize(b->stream);
	for(cudaGraphExec_t g : b->gexec)
		if(g) cudaGraphExecDestroy(g);
	for(cudaEvent_t e : b->join)
		if(e) cudaEventDestroy(e);
	if(b->fork) cudaEventDestroy(b->fork);
	if(b->done) cudaEventDestroy(b->done);
	if(b->stream) cudaStreamDestroy(b->stream);
	if(b->xstream)
		cudaStreamSynchronize(b->xstream);
	if(b->d_kinds) cudaFree(b->d_kinds);
	if(b->d_units) cudaFree(b->d_units);
	if(b->d_ctr) cudaFree(b->d_ctr);
	for(size_t k = 1; k < b->fspec.size(); k++)
		for(void *p : b->fspec[k])
			if(p) cudaFree(p);
	for(cudaEvent_t e : b->fdone)
		if(e) cudaEventDestroy(e);
	for(cudaEvent_t e : b->xdone)
		if(e) cudaEventDestroy(e);
	if(b->xstream) cudaStreamDestroy(b->xstream);
	for(fxb_ctx *c : b->m)
		c->batched = false;
	delete b;
}

#define BK(b, call)                                                          \
	do {                                                                     \
		cudaError_t e_ = (call);                                             \
		if(e_ != cudaSuccess)                                                \
		{                                                                    \
			(b)->err = std::string(#call) + ": " + cudaGetErrorString(e_);   \
			return e_ == cudaErrorMemoryAllocation ? FXB_ERR_NOMEM : FXB_ERR_CUDA; \
		}                                                                    \
	} while(0)

// Whether the members allow the fused launches (see fxb_batch_set_fused):
// every F kind a tensor-core FFT kind or a persistent one.
static bool batch_fusable(const fxb_batch *b)
{
	if(!b->fused || b->m.size() > (size_t)kFsMultiMembers)
		return false;
	for(const fxb_ctx *c : b->m)
	{
		if(!c->tc || c->f8 || !c->pclass.empty() || c->nzoom || c->nraw)
			return false;
		for(const FKind &k : c->fkinds)
			if(!k.tcfft && !k.persist)
				return false;
	}
	return true;
}

// The fused F launch's work list: the members' own lists, class by class
// (wide units of all members first), each member's kinds renumbered.
static fxb_status batch_fused_plan(fxb_batch *b)
{
	if(b->d_units)
		return FXB_OK;
	std::vector<FsMultiKind> kinds;
	std::vector<int> k0(b->m.size());
	for(size_t i = 0; i < b->m.size(); i++)
	{
		k0[i] = (int)kinds.size();
		for(FsMultiKind mk : b->m[i]->pkinds)
		{
			mk.member = (int32_t)i;
			kinds.push_back(mk);
		}
	}
	std::vector<FsMultiUnit> units;
	for(int cl = 0; cl < kFsMultiClasses; cl++)
	{
		b->unit0[cl] = (int32_t)units.size();
		for(size_t i = 0; i < b->m.size(); i++)
		{
			const fxb_ctx *c = b->m[i];
			for(int u = c->punit0[cl]; u < c->punit0[cl] + c->pnunit[cl]; u++)
			{
				FsMultiUnit w = c->punits[u];
				w.kind += k0[i];
				units.push_back(w);
			}
		}
		b->nunit[cl] = (int32_t)units.size() - b->unit0[cl];
	}
	BK(b, cudaMalloc(&b->d_kinds, sizeof(FsMultiKind) * std::max<size_t>(kinds.size(), 1)));
	BK(b, cudaMalloc(&b->d_units, sizeof(FsMultiUnit) * std::max<size_t>(units.size(), 1)));
	BK(b, cudaMalloc(&b->d_ctr, kFsMultiClasses * sizeof(int32_t)));
	if(!kinds.empty())
		BK(b, cudaMemcpy(b->d_kinds, kinds.data(), sizeof(FsMultiKind) * kinds.size(), cudaMemcpyHostToDevice));
	if(!units.empty())
		BK(b, cudaMemcpy(b->d_units, units.data(), sizeof(FsMultiUnit) * units.size(), cudaMemcpyHostToDevice));
	const size_t nslot = b->gexec.size();
	b->fspec.assign(nslot, std::vector<void *>(b->m.size(), nullptr));
	b->ftmap.assign(nslot, std::vector<std::vector<TmapBytes>>(b->m.size()));
	BK(b, cudaStreamCreateWithFlags(&b->xstream, cudaStreamNonBlocking));
	b->fdone.assign(nslot, nullptr);
	b->xdone.assign(nslot, nullptr);
	for(size_t k = 0; k < nslot; k++)
	{
		BK(b, cudaEventCreateWithFlags(&b->fdone[k], cudaEventDisableTiming));
		BK(b, cudaEventCreateWithFlags(&b->xdone[k], cudaEventDisableTiming));
		for(size_t i = 0; i < b->m.size(); i++)
		{
			fxb_ctx *c = b->m[i];
			void *sp = c->d_specn;
			if(k > 0)
			{
				// times past T of every block stay zero
				BK(b, cudaMalloc(&sp, sizeof(uint32_t) * (size_t)c->specn_elems));
				b->fspec[k][i] = sp;
				BK(b, cudaMemset(sp, 0, sizeof(uint32_t) * (size_t)c->specn_elems));
			}
			else
				b->fspec[k][i] = sp;
			for(const auto &g : c->xgroups)
			{
				TmapBytes tm;
				memset(&tm, 0, sizeof(tm));
				if(k == 0)
					memcpy(&tm, g.tmap, sizeof(tm));
				else if(g.xmac && !tc_make_tensormap(&tm, (const uint32_t *)sp + g.spec_base, g.shape, g.nf))
				{
					b->err = "cuTensorMapEncodeTiled failed for a batch spectra buffer";
					return FXB_ERR_CUDA;
				}
				b->ftmap[k][i].push_back(tm);
			}
		}
	}
	return FXB_OK;
}

// The fused F part of one subint (slot k) on the batch stream: every
// member's preparation as a branch, then the members' tensor-core FFT kinds
// and the persistent F launches into slot k's spectra (each its own branch),
// then the members' weights as branches.
static void batch_fused_launch(fxb_batch *b, int k, const std::vector<Slot *> &slots, bool capture)
{
	const unsigned evf = capture ? cudaEventRecordExternal : cudaEventRecordDefault;
	const size_t n = b->m.size();
	cudaEventRecord(b->fork, b->stream);
	for(size_t i = 0; i < n; i++)
	{
		fxb_ctx *c = b->m[i];
		cudaStreamWaitEvent(c->stream, b->fork, 0);
		launch_prep(c, *slots[i], c->stream, evf);
	}
	for(size_t i = 0; i < n; i++)
	{
		cudaEventRecord(b->join[i], b->m[i]->stream);
		cudaStreamWaitEvent(b->stream, b->join[i], 0);
	}
	// the F launches as parallel branches: each member's tensor-core FFT kinds
	// on its own stream, the persistent class kernels on the streams of
	// members without such kinds (or on the batch stream), so that each fills
	// the others' tails
	FsMultiArgs ma;
	memset(&ma, 0, sizeof(ma));
	ma.kinds = b->d_kinds;
	ma.units = b->d_units;
	for(int cl = 0; cl < kFsMultiClasses; cl++)
	{
		ma.unit0[cl] = b->unit0[cl];
		ma.nunit[cl] = b->nunit[cl];
	}
	ma.ctr = b->d_ctr;
	cudaMemsetAsync(b->d_ctr, 0, kFsMultiClasses * sizeof(int32_t), b->stream);
	cudaEventRecord(b->fork, b->stream);
	std::vector<cudaStream_t> free_st;
	std::vector<char> used(n, 0);
	for(size_t i = 0; i < n; i++)
	{
		fxb_ctx *c = b->m[i];
		ma.m[i] = fs_args(c, *slots[i]);
		ma.m[i].spec = b->fspec[k][i];
		bool tc = false;
		for(const FKind &fk : c->fkinds)
			tc = tc || fk.tcfft;
		if(!tc)
		{
			free_st.push_back(c->stream);
			continue;
		}
		cudaStreamWaitEvent(c->stream, b->fork, 0);
		used[i] = 1;
		for(const FKind &fk : c->fkinds)
			if(fk.tcfft)
			{
				const cudaError_t le = launch_fstage_tc(fk, ma.m[i], c->nsm, c->stream);
				if(le != cudaSuccess && c->launch_err == cudaSuccess)
					c->launch_err = le;
			}
	}
	const size_t nps = std::min<size_t>(free_st.size(), 2 * kFsMultiClasses);
	free_st.resize(nps);
	for(size_t j = 0; j < n && nps; j++)
		if(!used[j] && std::find(free_st.begin(), free_st.end(), b->m[j]->stream) != free_st.end())
		{
			cudaStreamWaitEvent(b->m[j]->stream, b->fork, 0);
			used[j] = 1;
		}
	if(nps == 0)
		free_st.assign(1, b->stream);
	const cudaError_t le = launch_fstage_multi_on(ma, b->m[0]->nsm, free_st.data(), (int)free_st.size());
	if(le != cudaSuccess && b->m[0]->launch_err == cudaSuccess)
		b->m[0]->launch_err = le;
	for(size_t i = 0; i < n; i++)
		if(used[i])
		{
			cudaEventRecord(b->join[i], b->m[i]->stream);
			cudaStreamWaitEvent(b->stream, b->join[i], 0);
		}
	cudaEventRecord(b->fork, b->stream);
	for(size_t i = 0; i < n; i++)
	{
		fxb_ctx *c = b->m[i];
		cudaStreamWaitEvent(c->stream, b->fork, 0);
		launch_xmac_weights(c, *slots[i], c->stream, evf, false, false);
	}
	for(size_t i = 0; i < n; i++)
	{
		cudaEventRecord(b->join[i], b->m[i]->stream);
		cudaStreamWaitEvent(b->stream, b->join[i], 0);
	}
}

// The fused XMAC of slot k's spectra: one launch over every member's groups
// of the first group's rows (groups of other rows: a launch each).
static void batch_fused_xmac(fxb_batch *b, int k, cudaStream_t st)
{
	XMultiArgs xm;
	memset(&xm, 0, sizeof(xm));
	const TcShape *common = nullptr;
	for(size_t i = 0; i < b->m.size(); i++)
	{
		fxb_ctx *c = b->m[i];
		for(size_t gi = 0; gi < c->xgroups.size(); gi++)
		{
			const auto &g = c->xgroups[gi];
			if(!g.xmac)
				continue;
			const void *tm = &b->ftmap[k][i][gi];
			if(!common)
				common = &g.shape;
			if(g.shape.nrow != common->nrow || g.shape.h16 != common->h16 ||
			   !xmac_multi_add(&xm, tm, g.shape, c->d_plans, g.d_idx, g.nf, c->d_acc))
				launch_xmac_tc(tm, g.shape, c->d_plans, g.d_idx, g.nf, c->nsm, c->d_err, c->d_acc, st);
		}
	}
	if(common)
		launch_xmac_tc_multi(xm, *common, b->m[0]->nsm, b->m[0]->d_err, st);
}

// capture every member's kernels for slot k (fused, or as parallel branches)
static fxb_status batch_graph(fxb_batch *b, int k, const std::vector<Slot *> &slots, bool fused)
{
	const size_t n = b->m.size();
	bool ok = b->gexec[k] != nullptr && b->g_fused[k] == (int)fused;
	for(size_t i = 0; ok && i < n; i++)
		ok = b->g_valid[k][i] == b->m[i]->d_valid && b->g_stride[k][i] == b->m[i]->valid_stride &&
		     b->g_gen[k][i] == b->m[i]->gen;
	if(ok)
		return FXB_OK;
	if(b->gexec[k])
	{
		cudaGraphExecDestroy(b->gexec[k]);
		b->gexec[k] = nullptr;
	}
	// one fork for all members, then every join: the branches are independent
	BK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
	if(fused)
		batch_fused_launch(b, k, slots, true);
	else
	{
		cudaEventRecord(b->fork, b->stream);
		for(size_t i = 0; i < n; i++)
		{
			fxb_ctx *c = b->m[i];
			cudaStreamWaitEvent(c->stream, b->fork, 0);
			launch_compute(c, *slots[i], c->stream, true);
		}
		for(size_t i = 0; i < n; i++)
		{
			cudaEventRecord(b->join[i], b->m[i]->stream);
			cudaStreamWaitEvent(b->stream, b->join[i], 0);
		}
	}
	cudaGraph_t g = nullptr;
	cudaError_t e = cudaStreamEndCapture(b->stream, &g);
	if(e == cudaSuccess)
		e = cudaGraphInstantiate(&b->gexec[k], g, 0);
	if(g)
		cudaGraphDestroy(g);
	if(e != cudaSuccess)
	{
		cudaGetLastError();
		b->gexec[k] = nullptr;
		b->graphs = false;              // eager launches from now on
		return FXB_OK;
	}
	for(size_t i = 0; i < n; i++)
	{
		b->g_valid[k][i] = b->m[i]->d_valid;
		b->g_stride[k][i] = b->m[i]->valid_stride;
		b->g_gen[k][i] = b->m[i]->gen;
	}
	b->g_fused[k] = (int)fused;
	return FXB_OK;
}

fxb_batch *fxb_batch_create(fxb_ctx *const *members, int32_t n, fxb_status *status)
{
	auto fail = [&](fxb_status st) -> fxb_batch * {
		if(status) *status = st;
		return nullptr;
	};
	if(!members || n < 1)
		return fail(FXB_ERR_ARG);
	for(int i = 0; i < n; i++)
	{
		if(!members[i] || members[i]->batched || members[i]->slots.size() != members[0]->slots.size() ||
		   members[i]->next_slot != members[0]->next_slot || members[i]->device != members[0]->device)
			return fail(FXB_ERR_ARG);
		for(int j = 0; j < i; j++)
			if(members[j] == members[i])
				return fail(FXB_ERR_ARG);
	}
	fxb_batch *b = new fxb_batch;
	b->m.assign(members, members + n);
	const size_t nslot = members[0]->slots.size();
	b->gexec.assign(nslot, nullptr);
	b->g_valid.assign(nslot, std::vector<const uint8_t *>(n, nullptr));
	b->g_stride.assign(nslot, std::vector<int64_t>(n, 0));
	b->g_gen.assign(nslot, std::vector<int>(n, -1));
	b->g_fused.assign(nslot, -1);
	b->join.assign(n, nullptr);
	bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
	          cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
	          cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
	for(int i = 0; ok && i < n; i++)
		ok = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
	if(!ok)
	{
		free_batch(b);
		return fail(FXB_ERR_CUDA);
	}
	for(fxb_ctx *c : b->m)
		c->batched = true;
	if(status) *status = FXB_OK;
	return b;
}

static fxb_status batch_submit(fxb_batch *b, const fxb_member_subint *data, int32_t sec, int32_t ns, bool device)
{
	if(!b || !data)
		return FXB_ERR_ARG;
	const size_t n = b->m.size();
	// argument checks first, so that a rejected call stages nothing and the
	// members' slots stay in step
	for(size_t i = 0; i < n; i++)
	{
		const fxb_member_subint &d = data[i];
		if(!d.bufs || !d.nbytes || !d.datasec || !d.datans)
			return FXB_ERR_ARG;
		for(int s = 0; s < b->m[i]->S; s++)
		{
			if(!b->m[i]->delay_set[s])
			{
				b->err = "delay model not set for every station of every member";
				return FXB_ERR_STATE;
			}
			if(d.nbytes[s] < 0 || (d.nbytes[s] > 0 && !d.bufs[s]))
			{
				b->err = "bad station buffer";
				return FXB_ERR_ARG;
			}
		}
	}
	const int k = b->m[0]->next_slot;
	bool tuning = false;
	for(fxb_ctx *c : b->m)
		tuning = tuning || c->tune.iter < c->tune.total;
	const bool pipelined = !tuning && batch_fusable(b) && !b->fspec.empty();
	std::vector<Slot *> slots(n, nullptr);
	for(size_t i = 0; i < n; i++)
	{
		fxb_ctx *c = b->m[i];
		const fxb_member_subint &d = data[i];
		const fxb_status rc = stage_subint(c, d.bufs, d.nbytes, d.datasec, d.datans, d.validflags, sec, ns, device,
		                                   &slots[i]);
		if(rc != FXB_OK)
		{
			b->err = std::string("member ") + std::to_string(i) + ": " + c->err;
			return rc;
		}
		BK(b, cudaStreamWaitEvent(b->stream, slots[i]->copied, 0));
		// and after whatever the member's own stream still holds (a reset, a
		// read); a pipelined batch only when the member has enqueued any,
		// since that stream also waits for the last subint's XMAC
		if(!pipelined || c->dirty)
		{
			BK(b, cudaEventRecord(b->join[i], c->stream));
			BK(b, cudaStreamWaitEvent(b->stream, b->join[i], 0));
			c->dirty = false;
		}
	}
	// a member still tuning runs eagerly (one member after the other, so
	// that its launch times are its own)
	const bool fused = !tuning && batch_fusable(b);
	if(fused)
	{
		const fxb_status rc = batch_fused_plan(b);
		if(rc != FXB_OK)
			return rc;
	}
	if(b->graphs && !tuning)
	{
		const fxb_status rc = batch_graph(b, k, slots, fused);
		if(rc != FXB_OK)
			return rc;
	}
	// fused: slot k's spectra are free once the XMAC of its last subint is done
	if(fused)
		BK(b, cudaStreamWaitEvent(b->stream, b->xdone[k], 0));
	if(b->graphs && !tuning)
		BK(b, cudaGraphLaunch(b->gexec[k], b->stream));
	else if(fused)
		batch_fused_launch(b, k, slots, false);
	else
		for(size_t i = 0; i < n; i++)
			launch_compute(b->m[i], *slots[i], b->stream, false);
	cudaStream_t endst = b->stream;
	if(fused)
	{
		// the XMAC beside the next subint's F stage
		BK(b, cudaEventRecord(b->fdone[k], b->stream));
		BK(b, cudaStreamWaitEvent(b->xstream, b->fdone[k], 0));
		batch_fused_xmac(b, k, b->xstream);
		BK(b, cudaEventRecord(b->xdone[k], b->xstream));
		endst = b->xstream;
	}
	for(fxb_ctx *c : b->m)
		if(take_launch_err(c) != FXB_OK)
		{
			b->err = c->err;
			return FXB_ERR_CUDA;
		}
	for(fxb_ctx *c : b->m)
		if(c->tune.iter < c->tune.total)
			tune_collect(c);
	BK(b, cudaGetLastError());
	BK(b, cudaEventRecord(b->done, endst));
	for(size_t i = 0; i < n; i++)
	{
		BK(b, cudaEventRecord(slots[i]->done, endst));
		BK(b, cudaStreamWaitEvent(b->m[i]->stream, b->done, 0));
		slots[i]->tpending = b->m[i]->timing_on;
		b->m[i]->last_slot = (int)(slots[i] - b->m[i]->slots.data());
		b->m[i]->timed = true;
	}
	return FXB_OK;
}

fxb_status fxb_batch_submit(fxb_batch *b, const fxb_member_subint *data, int32_t sec, int32_t ns)
{
	return batch_submit(b, data, sec, ns, false);
}

fxb_status fxb_batch_submit_device(fxb_batch *b, const fxb_member_subint *data, int32_t sec, int32_t ns)
{
	return batch_submit(b, data, sec, ns, true);
}

fxb_status fxb_batch_sync(fxb_batch *b)
{
	if(!b)
		return FXB_ERR_ARG;
	BK(b, cudaStreamSynchronize(b->stream));
	if(b->xstream)
		BK(b, cudaStreamSynchronize(b->xstream));
	for(fxb_ctx *c : b->m)
	{
		const fxb_status st = check_device_error(c);
		if(st != FXB_OK)
		{
			b->err = c->err;
			return st;
		}
	}
	return FXB_OK;
}

fxb_status fxb_batch_autotune(fxb_batch *b, int32_t rounds)
{
	if(!b)
		return FXB_ERR_ARG;
	for(fxb_ctx *c : b->m)
	{
		const fxb_status st = fxb_autotune(c, rounds);
		if(st != FXB_OK)
		{
			b->err = c->err;
			return st;
		}
	}
	return FXB_OK;
}

fxb_status fxb_batch_set_graphs(fxb_batch *b, int32_t on)
{
	if(!b) return FXB_ERR_ARG;
	b->graphs = on != 0;
	return FXB_OK;
}

fxb_status fxb_batch_set_fused(fxb_batch *b, int32_t on, int32_t *fused)
{
	if(!b) return FXB_ERR_ARG;
	b->fused = on != 0;
	if(fused)
		*fused = batch_fusable(b) ? 1 : 0;
	return FXB_OK;
}

const char *fxb_batch_last_error(const fxb_batch *b) { return b ? b->err.c_str() : ""; }

fxb_status fxb_batch_get_stream(const fxb_batch *b, void **stream)
{
	if(!b || !stream) return FXB_ERR_ARG;
	*stream = (void *)b->stream;
	return FXB_OK;
}

void fxb_batch_destroy(fxb_batch *b)
{
	if(b)
		free_batch(b);
}

}  // extern "C"
