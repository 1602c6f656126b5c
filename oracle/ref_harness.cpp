/* Harness that drives the reference correlator's own compiled CPU hot path.
 *
 * Test infrastructure only (oracle): it links the reference's Configuration,
 * Model, Mode/Mk5Mode and mark5access objects built by oracle/Makefile.ref
 * and exposes a small C interface that the tests and the CPU baseline call
 * through ctypes.  Nothing in the product library links this file.
 *
 * What comes from the reference unchanged: .input/.calc/.im parsing, the
 * result layout (Configuration::populateResultLengths), the per-station
 * F stage (Mode::process, Mk5Mode::unpack, mark5access VDIF decoding) and the
 * delay interpolator (Model::calculateDelayInterpolator).
 *
 * What this file restates, because Core cannot be constructed without an MPI
 * job: the per-thread loop of Core::processdata (mpifxcorr/src/core.cpp:
 * 705-730 station set-up, 796-811 F-stage batches, 877-972 XMAC,
 * 998-1045 baseline weights) and the result merge of
 * Core::uvshiftAndAverageBaselineFreq (core.cpp:1774-1787, no-shift,
 * no-averaging branch), Core::averageAndSendAutocorrs (core.cpp:1266-1363)
 * and the baseline-weight copy (core.cpp:1068-1086).  Threads split the FFT
 * blocks of a subintegration into contiguous ranges as Core::updateconfig
 * does (core.cpp:2090-2095); each thread owns its own Mode objects.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <thread>
#include <mutex>
#include "configuration.h"
#include "mode.h"
#include "visibility.h"
#include "datamuxer.h"
#include "mk5mode.h"
#include "model.h"
#include "mark5access.h"
#include "vdiffile.h"
#include "fxb_config_adapter.h"
#include <dlfcn.h>
#include <pthread.h>

namespace {

struct RefJob
{
	Configuration *config;
	int numds, numbl, nfreq, blockspersend, nbuffered, corelen;
	std::vector<std::vector<Mode *> > modes;   // [thread][datastream]
};

/* Per-thread accumulators in the core-result layout (complex index space). */
struct ThreadAcc
{
	std::vector<cf32> results;
	std::vector<cf32> xc;        // full-resolution cross products, [f][b][p][nchan]
};

/* offset of (f, b) in the full-resolution thread buffer */
static int64_t xc_offset(Configuration *c, int nfreq, int numbl, int f, int b, int64_t *total)
{
	int64_t off = 0, want = -1;
	for(int ff = 0; ff < nfreq; ff++)
	{
		if(!c->isFrequencyUsed(0, ff)) continue;
		for(int bb = 0; bb < numbl; bb++)
		{
			int lf = c->getBLocalFreqIndex(0, bb, ff);
			if(lf < 0) continue;
			if(ff == f && bb == b) want = off;
			off += (int64_t)c->getBNumPolProducts(0, bb, lf) * c->getFNumChannels(ff);
		}
	}
	if(total) *total = off;
	return want;
}

Mode *make_mode(Configuration *c, int ds)
{
	Mode *m = c->getMode(0, ds);
	if(!m || !m->initialisedOK())
		return 0;
	return m;
}

void ensure_threads(RefJob *j, int nthreads)
{
	while((int)j->modes.size() < nthreads)
	{
		std::vector<Mode *> ms;
		for(int d = 0; d < j->numds; d++)
			ms.push_back(make_mode(j->config, d));
		j->modes.push_back(ms);
	}
}

/* One thread's share of Core::processdata for blocks [startblock, startblock+numblocks). */
void process_range(RefJob *j, int t, int startblock, int numblocks,
	const unsigned char *const *bufs, const int *nbytes, const int *dscan, const int *dsec, const int *dns,
	const int *const *validflags, int scan, int sec, int ns, ThreadAcc *acc)
{
	Configuration *config = j->config;
	std::vector<Mode *> &modes = j->modes[t];
	const int nbuf = j->nbuffered;
	f32 *fres = (f32 *)&acc->results[0];

	for(int d = 0; d < j->numds; d++)
	{
		modes[d]->zeroAutocorrelations();
		modes[d]->setValidFlags((s32 *)validflags[d]);
		modes[d]->setData((u8 *)bufs[d], nbytes[d], dscan[d], dsec[d], dns[d]);
		modes[d]->setOffsets(scan, sec, ns);
		modes[d]->setDumpKurtosis(false);
		if(config->getDPhaseCalIntervalMHz(0, d) > 0)
			modes[d]->resetpcal();              /* core.cpp:716-728 */
	}

	int numfftloops = numblocks / nbuf + ((numblocks % nbuf) ? 1 : 0);
	for(int fftloop = 0; fftloop < numfftloops; fftloop++)
	{
		for(int d = 0; d < j->numds; d++)
			for(int sub = 0; sub < nbuf; sub++)
			{
				int i = fftloop * nbuf + sub + startblock;
				if(i >= startblock + numblocks)
					break;
				modes[d]->process(i, sub);
			}

		/* XMAC (core.cpp:877-972): accumulate directly in core-result order;
		 * each element receives the same sequence of products as the
		 * reference's per-stride thread buffer. */
		for(int f = 0; f < j->nfreq; f++)
		{
			if(!config->isFrequencyUsed(0, f))
				continue;
			int nchan = config->getFNumChannels(f);
			for(int b = 0; b < j->numbl; b++)
			{
				int lf = config->getBLocalFreqIndex(0, b, f);
				if(lf < 0)
					continue;
				const Mode *m1 = modes[config->getBOrderedDataStream1Index(0, b)];
				const Mode *m2 = modes[config->getBOrderedDataStream2Index(0, b)];
				int64_t base = xc_offset(config, j->nfreq, j->numbl, f, b, 0);
				for(int sub = 0; sub < nbuf; sub++)
				{
					int i = fftloop * nbuf + sub + startblock;
					if(i >= startblock + numblocks)
						break;
					for(int p = 0; p < config->getBNumPolProducts(0, b, lf); p++)
					{
						const cf32 *v1 = m1->getFreqs(config->getBDataStream1BandIndex(0, b, lf, p), sub);
						const cf32 *v2 = m2->getConjugatedFreqs(config->getBDataStream2BandIndex(0, b, lf, p), sub);
						cf32 *a = &acc->xc[base + p * nchan];
						for(int l = 0; l < nchan; l++)
						{
							a[l].re += v1[l].re * v2[l].re - v1[l].im * v2[l].im;
							a[l].im += v1[l].re * v2[l].im + v1[l].im * v2[l].re;
						}
					}
				}
			}
		}

		/* baseline weights (core.cpp:998-1045) */
		for(int sub = 0; sub < nbuf; sub++)
		{
			int i = fftloop * nbuf + sub + startblock;
			if(i >= startblock + numblocks)
				break;
			for(int f = 0; f < j->nfreq; f++)
			{
				if(!config->isFrequencyUsed(0, f))
					continue;
				for(int b = 0; b < j->numbl; b++)
				{
					int lf = config->getBLocalFreqIndex(0, b, f);
					if(lf < 0)
						continue;
					const Mode *m1 = modes[config->getBOrderedDataStream1Index(0, b)];
					const Mode *m2 = modes[config->getBOrderedDataStream2Index(0, b)];
					int widx = config->getCoreResultBWeightOffset(0, f, b) * 2;
					for(int p = 0; p < config->getBNumPolProducts(0, b, lf); p++)
					{
						int r1 = config->getBDataStream1RecordBandIndex(0, b, lf, p);
						int r2 = config->getBDataStream2RecordBandIndex(0, b, lf, p);
						if(r1 < 0 || r2 < 0)
							continue;
						fres[widx + p] += m1->getDataWeight(r1, sub) * m2->getDataWeight(r2, sub);
					}
				}
			}
		}
	}

	/* thread results into the core layout with channel averaging
	 * (core.cpp:1774-1802: mean over chans-to-average channels) */
	for(int f = 0; f < j->nfreq; f++)
	{
		if(!config->isFrequencyUsed(0, f))
			continue;
		int nchan = config->getFNumChannels(f);
		int avg = config->getFChannelsToAverage(f);
		for(int b = 0; b < j->numbl; b++)
		{
			int lf = config->getBLocalFreqIndex(0, b, f);
			if(lf < 0)
				continue;
			int64_t src = xc_offset(config, j->nfreq, j->numbl, f, b, 0);
			int core = config->getCoreResultBaselineOffset(0, f, b);
			for(int p = 0; p < config->getBNumPolProducts(0, b, lf); p++)
				for(int k = 0; k < nchan / avg; k++)
				{
					const cf32 *x = &acc->xc[src + (int64_t)p * nchan + (int64_t)k * avg];
					if(avg == 1)
					{
						acc->results[core + p * nchan + k].re += x[0].re;
						acc->results[core + p * nchan + k].im += x[0].im;
					}
					else
					{
						f32 sr = 0.0f, si = 0.0f;
						for(int l = 0; l < avg; l++) { sr += x[l].re; si += x[l].im; }
						acc->results[core + (p * nchan) / avg + k].re += sr / avg;
						acc->results[core + (p * nchan) / avg + k].im += si / avg;
					}
				}
		}
	}

	/* autocorrelations and their weights (core.cpp:1266-1363) */
	bool writecross = modes[0]->writeCrossAutoCorrs() && config->getMaxProducts() > 2;
	for(int d = 0; d < j->numds; d++)
	{
		modes[d]->averageFrequency();
		int ridx = config->getCoreResultAutocorrOffset(0, d);
		for(int pass = 0; pass < (writecross ? 2 : 1); pass++)
			for(int k = 0; k < config->getDNumTotalBands(0, d); k++)
			{
				int fi = config->getDTotalFreqIndex(0, d, k);
				if(!(config->isFrequencyUsed(0, fi) || config->isEquivalentFrequencyUsed(0, fi)))
					continue;
				int fc = config->getFNumChannels(fi) / config->getFChannelsToAverage(fi);
				const cf32 *ac = modes[d]->getAutocorrelation(pass == 1, k);
				for(int l = 0; l < fc; l++)
				{
					acc->results[ridx + l].re += ac[l].re;
					acc->results[ridx + l].im += ac[l].im;
				}
				ridx += fc;
			}
		int widx = config->getCoreResultACWeightOffset(0, d) * 2;
		int nrec = config->getDNumRecordedBands(0, d);
		for(int pass = 0; pass < (writecross ? 2 : 1); pass++)
			for(int k = 0; k < config->getDNumTotalBands(0, d); k++)
			{
				int fi = config->getDTotalFreqIndex(0, d, k);
				if(!(config->isFrequencyUsed(0, fi) || config->isEquivalentFrequencyUsed(0, fi)))
					continue;
				if(k < nrec)
					fres[widx] += modes[d]->getWeight(false, k);
				else
				{
					/* a zoom band takes the weight of its parent band
					 * (core.cpp:1311-1322) */
					int lf = config->getDLocalZoomFreqIndex(0, d, k - nrec);
					int parent = config->getDZoomFreqParentFreqIndex(0, d, lf);
					for(int l = 0; l < nrec; l++)
						if(config->getDLocalRecordedFreqIndex(0, d, l) == parent &&
						   config->getDZoomBandPol(0, d, k - nrec) == config->getDRecordedBandPol(0, d, l))
							fres[widx] += modes[d]->getWeight(false, l);
				}
				widx++;
			}
	}

	/* phase-cal tones of the thread's blocks, band by band (core.cpp:1124-1150) */
	for(int d = 0; d < j->numds; d++)
	{
		if(config->getDPhaseCalIntervalMHz(0, d) <= 0)
			continue;
		modes[d]->finalisepcal();
		int ridx = config->getCoreResultPCalOffset(0, d);
		for(int b = 0; b < config->getDNumRecordedBands(0, d); b++)
		{
			int lf = config->getDLocalRecordedFreqIndex(0, d, b);
			for(int k = 0; k < config->getDRecordedFreqNumPCalTones(0, d, lf); k++)
			{
				acc->results[ridx].re += modes[d]->getPcal(b, k).re;
				acc->results[ridx].im += modes[d]->getPcal(b, k).im;
				ridx++;
			}
		}
	}
}

/* DataStream control blocks: VDIFDataStream::calculateControlParams over
 * DataStream::calculateControlParams (vdiffile.cpp:358-485,
 * datastream.cpp:376-636), run by the stock code on a ring whose segments
 * the caller describes the way the read thread fills them.  The VDIF muxer
 * parameters are set as VDIFDataStream::initialiseFile sets them
 * (vdiffile.cpp:520-545); the caller holds the locks of the current segment
 * and the next, as the datastream's main thread does. */
class RingVDIF : public VDIFDataStream
{
public:
	RingVDIF(const Configuration *c, int ds, int factor, int nseg, int *cid)
		: VDIFDataStream(c, ds, ds + 1, 1, cid, factor, nseg) {}
	void setup()
	{
		initialise();
		datastatuses = new MPI_Status[maxsendspersegment];
		controlstatuses = new MPI_Status[maxsendspersegment];
		const int ci = bufferinfo[0].configindex;
		configurevdifmux(&vm, config->getFrameBytes(ci, streamnum),
		                 (int)config->getFramesPerSecond(ci, streamnum) / config->getDNumMuxThreads(ci, streamnum),
		                 config->getDNumBits(ci, streamnum), config->getDNumMuxThreads(ci, streamnum),
		                 config->getDMuxThreadMap(ci, streamnum), nSort, nGap,
		                 VDIF_MUX_FLAG_RESPECTGRANULARITY | VDIF_MUX_FLAG_PROPAGATEVALIDITY);
		waitsegment = 0;
	}
	int sizes(int *out)
	{
		out[0] = readbytes;
		out[1] = bufferbytes;
		out[2] = bufferinfo[0].nsinc;
		out[3] = bufferinfo[0].sendbytes;
		out[4] = bufferinfo[0].controllength;
		out[5] = config->getGuardNS(0);
		return 0;
	}
	/* segs: per segment scan, seconds, ns, readto, validbytes */
	int control(const long long *segs, int at, int keep, int lastvalid, int scan, int sec, int ns, int *out, int nout)
	{
		for(int i = 0; i < numdatasegments; i++)
		{
			bufferinfo[i].scan = (int)segs[5 * i];
			bufferinfo[i].scanseconds = (int)segs[5 * i + 1];
			bufferinfo[i].scanns = (int)segs[5 * i + 2];
			bufferinfo[i].readto = segs[5 * i + 3] != 0;
			bufferinfo[i].validbytes = segs[5 * i + 4];
			bufferinfo[i].numsent = 0;
			pthread_mutex_destroy(&bufferlock[i]);
			pthread_mutex_init(&bufferlock[i], NULL);
		}
		atsegment = at;
		waitsegment = at;
		keepreading = keep != 0;
		lastvalidsegment = lastvalid;
		pthread_mutex_lock(&bufferlock[atsegment]);
		pthread_mutex_lock(&bufferlock[(atsegment + 1) % numdatasegments]);
		const int bufferindex = calculateControlParams(scan, sec, ns);
		pthread_mutex_unlock(&bufferlock[atsegment]);
		pthread_mutex_unlock(&bufferlock[(atsegment + 1) % numdatasegments]);
		const s32 *cb = bufferinfo[atsegment].controlbuffer[0];
		const int n = bufferinfo[atsegment].controllength;
		if(nout < 2 + n)
			return -1;
		out[0] = bufferindex;
		out[1] = atsegment;
		for(int k = 0; k < n; k++)
			out[2 + k] = cb[k];
		return 2 + n;
	}
};

} // namespace

extern "C" {

/* Parse a .input file (with its .calc/.im) and build Mode objects for
 * nthreads threads.  Returns 0 when the reference rejects the job. */
void *dref_open(const char *inputfile, int nthreads)
{
	Configuration *c = new Configuration(inputfile, 0, 0.0);
	if(!c->consistencyOK())
	{
		delete c;
		return 0;
	}
	RefJob *j = new RefJob;
	j->config = c;
	j->numds = c->getNumDataStreams();
	j->numbl = c->getNumBaselines();
	j->nfreq = c->getFreqTableLength();
	j->blockspersend = c->getBlocksPerSend(0);
	j->nbuffered = c->getNumBufferedFFTs(0);
	j->corelen = c->getCoreResultLength(0);
	ensure_threads(j, nthreads < 1 ? 1 : nthreads);
	for(size_t t = 0; t < j->modes.size(); t++)
		for(int d = 0; d < j->numds; d++)
			if(!j->modes[t][d])
			{
				delete c;
				delete j;
				return 0;
			}
	return j;
}

void dref_close(void *h)
{
	RefJob *j = (RefJob *)h;
	if(!j) return;
	for(size_t t = 0; t < j->modes.size(); t++)
		for(size_t d = 0; d < j->modes[t].size(); d++)
			fxb_delete_mode(j->modes[t][d]);
	delete j->config;
	delete j;
}

/* info[0..5] = coreresultlength (complex), blockspersend, numdatastreams,
 * numbaselines, numbufferedffts, maxproducts */
void dref_info(void *h, int *info)
{
	RefJob *j = (RefJob *)h;
	info[0] = j->corelen;
	info[1] = j->blockspersend;
	info[2] = j->numds;
	info[3] = j->numbl;
	info[4] = j->nbuffered;
	info[5] = j->config->getMaxProducts();
}

/* Core-result offsets for layout parity: out[f*numbl + b] = baseline offset
 * (or -1), then bweight offsets likewise, then per-datastream autocorr,
 * acweight and phase-cal (-1 without phase cal) offsets.  out must hold
 * 2*nfreq*numbl + 3*numds ints. */
void dref_layout(void *h, int *out)
{
	RefJob *j = (RefJob *)h;
	Configuration *c = j->config;
	int k = 0;
	for(int pass = 0; pass < 2; pass++)
		for(int f = 0; f < j->nfreq; f++)
			for(int b = 0; b < j->numbl; b++)
			{
				if(!c->isFrequencyUsed(0, f) || c->getBLocalFreqIndex(0, b, f) < 0)
					out[k++] = -1;
				else
					out[k++] = pass == 0 ? c->getCoreResultBaselineOffset(0, f, b) : c->getCoreResultBWeightOffset(0, f, b);
			}
	for(int d = 0; d < j->numds; d++)
		out[k++] = c->getCoreResultAutocorrOffset(0, d);
	for(int d = 0; d < j->numds; d++)
		out[k++] = c->getCoreResultACWeightOffset(0, d);
	for(int d = 0; d < j->numds; d++)
		out[k++] = c->getDPhaseCalIntervalMHz(0, d) > 0 ? c->getCoreResultPCalOffset(0, d) : -1;
}

/* Correlate one subintegration and ADD it into coreresult (2*corelen floats).
 * bufs/nbytes/dscan/dsec/dns/validflags are per datastream, as the
 * DataStream control block would deliver them. */
int dref_process_subint(void *h, int nthreads,
	const unsigned char *const *bufs, const int *nbytes, const int *dscan, const int *dsec, const int *dns,
	const int *const *validflags, int scan, int sec, int ns, float *coreresult)
{
	RefJob *j = (RefJob *)h;
	if(nthreads < 1) nthreads = 1;
	ensure_threads(j, nthreads);
	std::vector<ThreadAcc> accs(nthreads);
	std::vector<std::thread> th;
	int bps = j->blockspersend;
	for(int t = 0; t < nthreads; t++)
	{
		/* contiguous split as Core::updateconfig (core.cpp:2090-2095) */
		int start = t * (bps / nthreads) + (t < bps % nthreads ? t : bps % nthreads);
		int num = bps / nthreads + (t < bps % nthreads ? 1 : 0);
		accs[t].results.assign(j->corelen, cf32{0.0f, 0.0f});
		{
			int64_t tot = 0;
			xc_offset(j->config, j->nfreq, j->numbl, -1, -1, &tot);
			accs[t].xc.assign(tot, cf32{0.0f, 0.0f});
		}
		if(nthreads == 1)
			process_range(j, 0, start, num, bufs, nbytes, dscan, dsec, dns, validflags, scan, sec, ns, &accs[0]);
		else
			th.emplace_back(process_range, j, t, start, num, bufs, nbytes, dscan, dsec, dns, validflags, scan, sec, ns, &accs[t]);
	}
	for(auto &x : th)
		x.join();
	for(int t = 0; t < nthreads; t++)
	{
		const float *src = (const float *)&accs[t].results[0];
		for(int i = 0; i < 2 * j->corelen; i++)
			coreresult[i] += src[i];
	}
	return 0;
}

/* Run Mode::process for one FFT of one datastream and return what the XMAC
 * would read: spectra[band][nchan] complex (all recorded bands), the data
 * weight, and the Mode's running autocorrelations after this FFT. */
int dref_mode_fft(void *h, int ds, const unsigned char *buf, int nbytes, int dscan, int dsec, int dns,
	const int *validflags, int scan, int sec, int ns, int fftindex, float *spectra, float *weight, float *autocorr)
{
	RefJob *j = (RefJob *)h;
	Configuration *c = j->config;
	Mode *m = j->modes[0][ds];
	m->zeroAutocorrelations();
	m->setValidFlags((s32 *)validflags);
	m->setData((u8 *)buf, nbytes, dscan, dsec, dns);
	m->setOffsets(scan, sec, ns);
	m->process(fftindex, 0);
	int nb = c->getDNumRecordedBands(0, ds);
	int nchan = c->getFNumChannels(c->getDTotalFreqIndex(0, ds, 0));
	for(int b = 0; b < nb; b++)
	{
		memcpy(spectra + (size_t)2 * b * nchan, m->getFreqs(b, 0), sizeof(float) * 2 * nchan);
		if(autocorr)
			memcpy(autocorr + (size_t)2 * b * nchan, m->getAutocorrelation(false, b), sizeof(float) * 2 * nchan);
	}
	*weight = m->getDataWeight(0, 0);
	return nb;
}

/* Delay interpolator exactly as Mode::setOffsets obtains it (mode.cpp:1541-1549). */
int dref_interpolator(void *h, int ds, int scan, int sec, int ns, double *coeffs)
{
	RefJob *j = (RefJob *)h;
	Configuration *c = j->config;
	Model *model = c->getModel();
	int nchan = c->getFNumChannels(c->getDTotalFreqIndex(0, ds, 0));
	double bw = c->getDRecordedBandwidth(0, ds, 0);
	double sampletime = 1.0 / (2.0 * bw);
	double timespan = j->blockspersend * 2 * nchan * sampletime / 1e6;
	int srcindex = model->getNumPhaseCentres(scan) == 1 ? 1 : 0;
	bool ok = model->calculateDelayInterpolator(scan, (double)sec + ns / 1e9, timespan, j->blockspersend,
		c->getDModelFileIndex(0, ds), srcindex, 2, coeffs);
	int intclockseconds = int(floor(c->getDClockCoeff(0, ds, 0) / 1000000.0 + 0.5));
	coeffs[2] -= 1000000 * intclockseconds;
	return ok ? 0 : -1;
}

/* Direct mark5access decode of nsamp samples per channel starting at
 * offsetsamples, the call Mk5Mode::unpack makes (mk5mode.cpp:119).  out is
 * [nchan][nsamp].  Returns mark5access's good-sample count. */
int dref_unpack(const char *formatname, const unsigned char *data, int offsetsamples, int nsamp, float *out)
{
	struct mark5_stream *ms = new_mark5_stream(new_mark5_stream_unpacker(0), new_mark5_format_generic_from_string(formatname));
	if(!ms)
		return -1000000;
	std::vector<float *> ptrs(ms->nchan);
	for(int c = 0; c < ms->nchan; c++)
		ptrs[c] = out + (size_t)c * nsamp;
	int good = mark5_unpack_with_offset(ms, data, offsetsamples, &ptrs[0], nsamp);
	delete_mark5_stream(ms);
	return good;
}

/* The reference's integration output: a Visibility for configuration 0 whose
 * integration starts at the start of scan 0 (visibility.cpp:46-117) takes the
 * nsub subint core results (2*corelen floats each) through addData, then
 * writedata() calibrates them and appends the SWIN records to
 * <OUTPUT FILENAME>/DIFX_<mjd>_<sec>.s0000.b0000 (visibility.cpp:348-900). */
int dref_visibility_write(void *h, const float *const *subints, int nsub)
{
	RefJob *j = (RefJob *)h;
	Configuration *c = j->config;
	static const std::string pnames[4] = {"RR", "LL", "RL", "LR"};
	const size_t nfl = 2 * (size_t)c->getMaxCoreResultLength();
	std::vector<char> disk(nfl * 4 * 2 + (1 << 20));
	Visibility v(c, 0, 1, disk.data(), (int)disk.size(), c->getExecuteSeconds(), 0, 0, 0, pnames);
	if(!v.configuredOK())
		return 1;
	std::vector<float> tmp(nfl);
	v.initialisePcalFiles();                 /* FxManager does this once (fxmanager.cpp:651) */
	for(int k = 0; k < nsub; k++)
	{
		memcpy(tmp.data(), subints[k], sizeof(float) * 2 * j->corelen);
		v.addData((cf32 *)tmp.data());
	}
	v.writedata();
	return 0;
}

/* The reference's INTERLACEDVDIF muxer on one read (VDIFMuxer,
 * datamuxer.cpp:106-848): inbytes of iframebytes-byte frames of the threads
 * tmap[nthreads] go through initialise, deinterlace and multiplex; out
 * receives the single-thread frames.  Returns the bytes written, or -1 when
 * the reference rejects the read. */
int dref_vdif_mux(const unsigned char *in, int inbytes, int nthreads, const int *tmap, int iframebytes, int fps,
                  int nbits, unsigned char *out)
{
	const int rframes = inbytes / iframebytes;
	VDIFMuxer m(0, 0, 0, nthreads, iframebytes, rframes, fps, nbits, (int *)tmap);
	DataMuxer *dm = &m;                    // the public interface (VDIFMuxer's overrides are protected)
	memcpy(dm->getCurrentDemuxBuffer(), in, (size_t)inbytes);
	if(!dm->initialise() || !dm->deinterlace(inbytes))
		return -1;
	return dm->multiplex(out);
}

} // extern "C"

extern "C" {

/* A datastream of the job with nseg segments of readbytes = factor / nseg *
 * (the largest subint's bytes); out: readbytes, bufferbytes, nsinc,
 * sendbytes, control words per subint, guard ns. */
void *dref_ds_create(void *h, int ds, int factor, int nseg, int *out)
{
	RefJob *j = (RefJob *)h;
	static int cid[1] = {1};
	RingVDIF *d = new RingVDIF(j->config, ds, factor, nseg, cid);
	d->setup();
	d->sizes(out);
	return d;
}

int dref_ds_control(void *d, const long long *segs, int at, int keep, int lastvalid, int scan, int sec, int ns,
                    int *out, int nout)
{
	return ((RingVDIF *)d)->control(segs, at, keep, lastvalid, scan, sec, ns, out, nout);
}

void dref_ds_destroy(void *d)
{
	(void)d;   /* the stock destructor closes files and frees MPI state it never opened here: leak the test object */
}

}

/* ---- the integration flow: Configuration -> fxb200 C ABI ---------------- */

extern "C" {

/* The fxb_job_desc of configuration 0, built by fxb_desc_from_configuration
 * from the stock Configuration; it stays valid until the process exits.
 * Returns null with err filled for a configuration outside the ABI. */
const void *dref_fxb_desc(void *h, int xmac_kind, char *err, int errlen)
{
	RefJob *j = (RefJob *)h;
	static std::vector<FxbConfigDesc *> keep;    // one per call, kept until the process exits
	FxbConfigDesc *d = new FxbConfigDesc;
	std::string e;
	if(!fxb_desc_from_configuration(j->config, 0, xmac_kind, *d, e))
	{
		snprintf(err, errlen, "%s", e.c_str());
		delete d;
		return 0;
	}
	keep.push_back(d);
	return &d->desc;
}

/* Each datastream's delay interpolator for (scan, sec, ns), from the stock
 * Model as Mode::setOffsets obtains it; returns the datastreams without one. */
int dref_fxb_interpolators(void *h, int scan, int sec, int ns, double *interp)
{
	RefJob *j = (RefJob *)h;
	return fxb_interpolators_from_model(j->config, 0, scan, sec, ns, interp);
}

/* What an integration into mpifxcorr does per configuration, written against
 * the product library's C ABI (loaded from libpath): the descriptor from the
 * Configuration, a context, then per subint k the interpolators from the
 * Model and fxb_submit_subint_interp with the datastreams' buffers
 * bufs[k * nds + ds]; finally fxb_read_results into coreresult (2 corelen
 * floats).  Returns 0, or -1 with err filled. */
int dref_fxb_correlate(void *h, const char *libpath, int xmac_kind, int nsub, const unsigned char *const *bufs,
                       const long long *nbytes, const int *datasec, const int *datans, const int *sec, const int *ns,
                       float *coreresult, long long nfloats, char *err, int errlen)
{
	RefJob *j = (RefJob *)h;
	typedef fxb_ctx *(*create_t)(const fxb_job_desc *, fxb_status *);
	typedef fxb_status (*submit_t)(fxb_ctx *, const uint8_t *const *, const int64_t *, const int32_t *,
	                               const int32_t *, const int32_t *const *, int32_t, int32_t, const double *);
	typedef fxb_status (*read_t)(fxb_ctx *, float *, size_t);
	typedef void (*destroy_t)(fxb_ctx *);
	typedef const char *(*lasterr_t)(const fxb_ctx *);
	void *lib = dlopen(libpath, RTLD_NOW | RTLD_LOCAL);
	if(!lib)
	{
		snprintf(err, errlen, "dlopen: %s", dlerror());
		return -1;
	}
	create_t fxb_create_p = (create_t)dlsym(lib, "fxb_create");
	submit_t fxb_submit_subint_interp_p = (submit_t)dlsym(lib, "fxb_submit_subint_interp");
	read_t fxb_read_results_p = (read_t)dlsym(lib, "fxb_read_results");
	destroy_t fxb_destroy_p = (destroy_t)dlsym(lib, "fxb_destroy");
	lasterr_t fxb_last_error_p = (lasterr_t)dlsym(lib, "fxb_last_error");
	if(!fxb_create_p || !fxb_submit_subint_interp_p || !fxb_read_results_p || !fxb_destroy_p || !fxb_last_error_p)
	{
		snprintf(err, errlen, "missing fxb200 entry points");
		return -1;
	}

	FxbConfigDesc d;
	std::string e;
	if(!fxb_desc_from_configuration(j->config, 0, xmac_kind, d, e))
	{
		snprintf(err, errlen, "%s", e.c_str());
		return -1;
	}
	fxb_status st = FXB_OK;
	fxb_ctx *ctx = fxb_create_p(&d.desc, &st);
	if(!ctx)
	{
		snprintf(err, errlen, "fxb_create: %d %s", (int)st, fxb_last_error_p(0));
		return -1;
	}
	const int nds = j->numds;
	std::vector<double> interp(3 * nds);
	std::vector<int64_t> nb(nds);
	for(int k = 0; k < nsub && st == FXB_OK; k++)
	{
		fxb_interpolators_from_model(j->config, 0, 0, sec[k], ns[k], interp.data());
		for(int ds = 0; ds < nds; ds++)
			nb[ds] = nbytes[k * nds + ds];
		st = fxb_submit_subint_interp_p(ctx, bufs + (size_t)k * nds, nb.data(), datasec + (size_t)k * nds,
		                                datans + (size_t)k * nds, 0, sec[k], ns[k], interp.data());
	}
	if(st == FXB_OK)
		st = fxb_read_results_p(ctx, coreresult, (size_t)nfloats);
	if(st != FXB_OK)
		snprintf(err, errlen, "fxb200: %d %s", (int)st, fxb_last_error_p(ctx));
	fxb_destroy_p(ctx);
	return st == FXB_OK ? 0 : -1;
}

}

