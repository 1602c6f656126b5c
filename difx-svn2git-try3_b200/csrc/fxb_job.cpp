// Job validation and the core-result layout.
//
// The layout restates Configuration::populateResultLengths
// (mpifxcorr/src/configuration.cpp:2212-2440) for one configuration with one
// phase centre, no pulsar bins and no phase cal: cross correlations
// [freq][baseline][product][nchan/avg], then baseline weights (products/2
// rounded up complex slots), then per datastream the autocorrelations of its
// recorded and then its zoom bands (parallel hands, then cross hands when the
// job has more than two products), then the autocorrelation weights.
//
// A zoom band is a channel window of a recorded band (mode.cpp:169-208).  Its
// frequency gets an XMAC plan of its own whose spectra rows are copied from
// the parent bands' spectra, so that stations whose zoom bands have different
// parents (a 16 MHz band of one station zoomed onto an 8 MHz band of another)
// correlate like any other frequency.

#include <algorithm>
#include <cmath>
#include <cstring>

#include "fxb_internal.h"

namespace fxb {

// calcstridelength (configuration.cpp:46-58): the array stride used by
// Mode's rotator tables; it enters the order-2 fringe phase.
int calcstridelength(unsigned int arraylength)
{
	if(arraylength <= 16)
		return (int)arraylength;
	for(unsigned int guess = (unsigned int)std::sqrt(arraylength + 0.1); ; --guess)
		if(arraylength % guess == 0)
			return (int)(arraylength / guess);
}

static bool fail(std::string &err, fxb_status &st, fxb_status code, const std::string &msg)
{
	err = msg;
	st = code;
	return false;
}

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// ------------------------------------------------------------------ phase cal
// Greatest common divisor of doubles rounded to integers (mathutil.cpp:8-30).
static long long gcd_rounded(double a, double b)
{
	long x = (long)std::floor(a + 0.5), y = (long)std::floor(b + 0.5);
	if(x == 0 || y == 0)
		return std::max(x, y);
	while(y != 0)
	{
		const long r = x % y;
		x = y;
		y = r;
	}
	return x;
}

// Comb tones from offset up to the band edge, a tone on both edges counted
// once (PCal::calcNumTones, pcal.cpp:205-222).
static int comb_tones(double bw, double offset, double step)
{
	if(bw <= 0.0 || step <= 0.0)
		return 0;
	int n = 0;
	double f = offset;
	while(f <= bw)
	{
		n++;
		f += step;
	}
	if(offset == 0.0 && f - step == bw)
		n--;
	return n;
}

constexpr int kMaxPcalBins = 32768;

// One recorded band's tones and extractor: the comb tones of the band
// (configuration.cpp:1776-1846) and, for the extractor PCal::getNew picks
// (pcal.cpp:139-191, with Mode's 1 MHz minimum frequency resolution), the
// bin count and tone bins of the implicit-shift extractor
// (pcal.cpp:927-958, 1073-1086) or of the shifting one (pcal.cpp:494-705).  A band without a tone reads as one zero
// tone (the dummy extractor).
static bool pcal_band(const fxb_freq &f, float interval, float base, Job::PcalBand &pb, std::string &err,
                      fxb_status &st)
{
	pb.nbins = pb.first = pb.step = pb.shift = 0;
	pb.fs = (int64_t)(2e6 * f.bw_mhz + 0.5);
	pb.tonefreq = 0.0;
	pb.lsb = f.lower_sideband ? 1 : 0;
	const double lo = f.freq_mhz, bw = f.bw_mhz;
	double tonefreq = (double)((int)(lo / interval)) * interval;
	int n = 0;
	if(f.lower_sideband)
	{
		// tones below the LO, counted downwards; the extraction is the same, the
		// tones lying at the same baseband offsets (configuration.cpp:1776-1811)
		if(tonefreq == lo)
			tonefreq -= interval;
		if(tonefreq >= lo - bw)
			while(tonefreq - (float)(n * interval) >= lo - bw)
				n++;
	}
	else
	{
		if(tonefreq <= lo)
			tonefreq += interval;
		if(tonefreq <= lo + bw)
			while(tonefreq + (float)(n * interval) <= lo + bw)
				n++;
	}
	if(n == 0)
	{
		pb.ntones = 1;
		return true;
	}
	pb.ntones = n;
	pb.tonefreq = tonefreq;
	int off;
	if(f.lower_sideband)
	{
		const double tone0 = 1e6 * tonefreq - 0 * 1e6 * interval - 1e6 * base;
		off = (int)(long)(1e6 * lo - tone0 + 0.5);
	}
	else
	{
		const double tone0 = 1e6 * tonefreq + 0 * 1e6 * interval + 1e6 * base;
		off = (int)(long)(tone0 - 1e6 * lo + 0.5);
	}
	const double fs = 2.0 * 1e6 * bw, sp = 1e6 * interval;
	int nbins = (int)(fs / gcd_rounded(fs, (double)off));
	const int nspacing = (int)(fs / gcd_rounded(fs, sp));
	const int nt = comb_tones(1e6 * bw, (double)off, sp);
	while(fs / (2 * nbins) > 1e6)
		nbins *= 2;
	if(nt == 0)
		return true;
	if(off == 0)
		return fail(err, st, FXB_ERR_UNSUPPORTED, "phase-cal comb needs the trivial extractor");
	if(nt != n)
		return fail(err, st, FXB_ERR_UNSUPPORTED, "phase-cal tone count differs between extractor and configuration");
	if(nbins % nspacing != 0)
	{
		// the shifting extractor (pcal.cpp:494-705): samples rotated by the
		// offset, folded into fs / gcd(fs, spacing) bins, tones at multiples of
		// the step from bin 0
		const int N = (int)(fs / gcd_rounded(fs, sp));
		const int stp = (int)std::floor(N * (sp / fs));
		if((int64_t)(nt - 1) * stp >= N)
			return fail(err, st, FXB_ERR_UNSUPPORTED, "phase-cal tones beyond the shifting extractor's bins");
		if(N > kMaxPcalBins)
			return fail(err, st, FXB_ERR_UNSUPPORTED, "phase-cal comb repeats after too many samples");
		pb.nbins = N;
		pb.step = stp;
		pb.first = 0;
		pb.shift = off;
		return true;
	}
	if(nbins > kMaxPcalBins)
		return fail(err, st, FXB_ERR_UNSUPPORTED, "phase-cal offset repeats after too many samples");
	pb.nbins = nbins;
	pb.step = (int)std::floor((double)nbins * (sp / fs));
	pb.first = (int)std::floor((double)nbins * ((double)off / fs));
	return true;
}

bool build_job(const fxb_job_desc *d, Job &job, std::string &err, fxb_status &st)
{
	st = FXB_OK;
	if(!d || d->nfreq <= 0 || !d->freqs || d->nstation < 1 || !d->stations || d->nbaseline < 0)
		return fail(err, st, FXB_ERR_ARG, "empty or null job description");
	if(d->nstation > kMaxStations)
		return fail(err, st, FXB_ERR_UNSUPPORTED, "too many stations");
	if(d->fringe_rot_order < 0 || d->fringe_rot_order > 2)
		return fail(err, st, FXB_ERR_ARG, "fringe rotation order must be 0, 1 or 2");
	if(d->xmac_kind < FXB_XMAC_FP32 || d->xmac_kind > FXB_XMAC_FP16)
		return fail(err, st, FXB_ERR_ARG, "unknown xmac kind");
	job.freqs.assign(d->freqs, d->freqs + d->nfreq);
	for(auto &f : job.freqs)
	{
		if(!(f.bw_mhz > 0.0) || f.nchan <= 0 || f.chans_to_avg <= 0 || f.nchan % f.chans_to_avg)
			return fail(err, st, FXB_ERR_ARG, "bad frequency entry");
		if(!is_pow2(f.nchan) || f.nchan < 16 || f.nchan > 8192)
			return fail(err, st, FXB_ERR_UNSUPPORTED, "channel counts must be powers of two in [16, 8192]");
	}
	for(int s = 0; s < d->nstation; s++)
	{
		const fxb_station &in = d->stations[s];
		Job::Station o;
		o.nbits = in.nbits;
		o.payload = in.payload_bytes;
		o.header = in.header_bytes;
		o.nband = in.nband;
		if(in.nband < 1 || in.nband > kMaxBandsPerStation || !in.band_freq || !in.band_pol)
			return fail(err, st, FXB_ERR_ARG, "station needs at least one band");
		if(!is_pow2(in.nband))
			return fail(err, st, FXB_ERR_UNSUPPORTED, "VDIF channel count must be a power of two");
		if(in.nbits == 2)
		{
			if(in.nband > 64)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "2-bit VDIF supports up to 64 channels");
		}
		else if(in.nbits == 8)
		{
			if(in.nband > 4)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "8-bit VDIF supports up to 4 channels");
		}
		else
			return fail(err, st, FXB_ERR_UNSUPPORTED, "only 2-bit and 8-bit samples are supported");
		if(in.header_bytes != 32 && in.header_bytes != 16)
			return fail(err, st, FXB_ERR_ARG, "VDIF header must be 16 or 32 bytes");
		if(in.payload_bytes <= 0 || in.payload_bytes % 8 || ((int64_t)in.payload_bytes * 8) % (in.nbits * in.nband))
			return fail(err, st, FXB_ERR_ARG, "payload must be a multiple of 8 bytes holding whole samples");
		o.band_freq.assign(in.band_freq, in.band_freq + in.nband);
		o.band_pol.assign(in.band_pol, in.band_pol + in.nband);
		for(int b = 0; b < in.nband; b++)
			if(o.band_freq[b] < 0 || o.band_freq[b] >= d->nfreq)
				return fail(err, st, FXB_ERR_ARG, "band frequency index out of range");
		// corrections of each band's recorded frequency (configuration.cpp:1641-1672)
		{
			const double *src[4] = {in.band_clock_us, in.band_clock_delta_us, in.band_phase_deg, in.band_lo_offset_hz};
			std::vector<double> *dst[4] = {&o.clk, &o.dclk, &o.phase, &o.looff};
			for(int q = 0; q < 4; q++)
			{
				dst[q]->assign(in.nband, 0.0);
				if(!src[q])
					continue;
				for(int b = 0; b < in.nband; b++)
				{
					const double v = src[q][b];
					if(!std::isfinite(v))
						return fail(err, st, FXB_ERR_ARG, "band corrections must be finite");
					(*dst[q])[b] = v;
					if(v != 0.0)
						o.has_corr = true;
					for(int c = 0; c < b; c++)
						if(o.band_freq[c] == o.band_freq[b] && (*dst[q])[c] != v)
							return fail(err, st, FXB_ERR_ARG, "bands of one frequency carry different corrections");
				}
			}
		}
		const fxb_freq &f0 = job.freqs[o.band_freq[0]];
		for(int b = 1; b < in.nband; b++)
		{
			const fxb_freq &fb = job.freqs[o.band_freq[b]];
			if(fb.nchan != f0.nchan || fb.bw_mhz != f0.bw_mhz)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "all bands of one station share bandwidth and channels");
		}
		if(in.nzoom < 0 || in.nzoom > kMaxBandsPerStation || (in.nzoom > 0 && (!in.zoom_freq || !in.zoom_pol)))
			return fail(err, st, FXB_ERR_ARG, "bad zoom band list");
		for(int z = 0; z < in.nzoom; z++)
		{
			const int zf = in.zoom_freq[z];
			if(zf < 0 || zf >= d->nfreq)
				return fail(err, st, FXB_ERR_ARG, "zoom frequency index out of range");
			// zoom frequencies come after the recorded ones (configuration.cpp:2598-2610)
			for(int b = 0; b < in.nband; b++)
				if(zf < o.band_freq[b])
					return fail(err, st, FXB_ERR_ARG, "a zoom frequency precedes a recorded frequency in the table");
			// parent: the last recorded frequency, in the station's order, whose
			// range holds the zoom band; offset in channels of the first recorded
			// frequency (configuration.cpp:1734-1754)
			const fxb_freq &zq = job.freqs[zf];
			const double lo = zq.freq_mhz - (zq.lower_sideband ? zq.bw_mhz : 0.0), hi = lo + zq.bw_mhz;
			int parent = -1, off = 0;
			for(int b = 0; b < in.nband; b++)
			{
				if(std::find(o.band_freq.begin(), o.band_freq.begin() + b, o.band_freq[b]) != o.band_freq.begin() + b)
					continue;
				const fxb_freq &pf = job.freqs[o.band_freq[b]];
				const double plo = pf.freq_mhz - (pf.lower_sideband ? pf.bw_mhz : 0.0), phi = plo + pf.bw_mhz;
				if(hi <= phi && lo >= plo)
				{
					parent = o.band_freq[b];
					off = (int)(((lo - plo) / f0.bw_mhz) * f0.nchan + 0.5);
				}
			}
			if(parent < 0)
				return fail(err, st, FXB_ERR_ARG, "zoom band outside every recorded band");
			const fxb_freq &pf = job.freqs[parent];
			if(std::fabs(zq.bw_mhz / zq.nchan - pf.bw_mhz / pf.nchan) > 1e-9)
				return fail(err, st, FXB_ERR_ARG, "zoom channel width differs from its parent's");
			// the parent band: the first recorded band of that frequency in the
			// zoom band's polarisation (configuration.cpp:1245-1258)
			int pb = -1;
			for(int b = 0; b < in.nband && pb < 0; b++)
				if(o.band_freq[b] == parent && o.band_pol[b] == in.zoom_pol[z])
					pb = b;
			if(pb < 0)
				return fail(err, st, FXB_ERR_ARG, "zoom band without a parent band of its polarisation");
			if(zq.lower_sideband || pf.lower_sideband)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "zoom bands of lower-sideband bands");
			if(off < 0 || off + zq.nchan > pf.nchan)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "zoom band channels outside its parent");
			// the zoom band's autocorrelation is the parent's, averaged by the
			// station's first recorded frequency (mode.cpp:389-397, 1399-1424):
			// the same as averaging the window itself only when the averaging
			// agrees and the window starts on an averaging boundary
			if(zq.chans_to_avg != f0.chans_to_avg || off % f0.chans_to_avg)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "zoom averaging differs from the station's recorded averaging");
			o.zoom_freq.push_back(zf);
			o.zoom_pol.push_back(in.zoom_pol[z]);
			o.zoom_parent.push_back(pb);
			o.zoom_choff.push_back(off);
		}
		if(!(in.pcal_interval_mhz >= 0.0) || !(in.pcal_base_mhz == in.pcal_base_mhz))
			return fail(err, st, FXB_ERR_ARG, "bad phase-cal interval");
		o.pcal_interval = (float)in.pcal_interval_mhz;
		o.pcal_base = (float)in.pcal_base_mhz;
		if(in.mux_threads < 0)
			return fail(err, st, FXB_ERR_ARG, "bad mux thread count");
		if(in.mux_threads > 0 && (in.mux_threads != in.nband || in.nbits != 2 || in.nband > 32 || in.nzoom > 0 ||
		                          o.pcal_interval > 0.0f))
			return fail(err, st, FXB_ERR_UNSUPPORTED,
			            "INTERLACEDVDIF needs one 2-bit band per thread, at most 32, without zoom bands or phase cal");
		o.mux_threads = in.mux_threads;
		if(in.complex_sampling)
		{
			// single-sideband complex sampling (mode.cpp:51-59, 889-905, 1155-1234);
			// 1-channel 2-bit complex data unpack in pairs of samples, whose edge
			// erasure Mk5Mode applies to the real arrays (mk5mode.cpp:129-147)
			if(in.complex_sampling != 1)
				return fail(err, st, FXB_ERR_ARG, "bad complex sampling kind");
			if(d->fringe_rot_order == 0)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "post-F fringe rotation of complex data (mode.cpp:1159-1162)");
			if((in.nbits == 2 && in.nband < 2) || (in.nbits == 8 && in.nband > 4) || in.mux_threads > 0 ||
			   in.nzoom > 0 || o.pcal_interval > 0.0f || f0.nchan < 32)
				return fail(err, st, FXB_ERR_UNSUPPORTED,
				            "complex sampling: 2-bit with 2..64 or 8-bit with 1..4 channels of at least 32 channels each, "
				            "without zoom bands, phase cal or INTERLACEDVDIF");
			if(((int64_t)in.payload_bytes * 8) % (2 * in.nbits * in.nband))
				return fail(err, st, FXB_ERR_ARG, "payload must hold whole complex samples");
			// an FFT window within 32 frames (the F stage's per-window frame mask)
			const int64_t fsamp = (int64_t)in.payload_bytes * 8 / (2 * in.nbits * in.nband);
			if((f0.nchan + fsamp - 1) / fsamp + 1 > 32)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "complex sampling: an FFT window spans more than 32 frames");
			o.cplx = true;
		}
		if(in.mux_raw)
		{
			// raw reads: thread frames of payload / threads bytes (whole 8-byte
			// VDIF units, so that every frame's payload words are aligned)
			if(in.mux_threads < 1 || in.header_bytes != 32 || in.payload_bytes % in.mux_threads ||
			   (in.payload_bytes / in.mux_threads) % 8)
				return fail(err, st, FXB_ERR_UNSUPPORTED,
				            "raw INTERLACEDVDIF reads need 32-byte headers and thread payloads of a multiple of 8 bytes");
			o.mux_raw = true;
			for(int t = 0; t < in.mux_threads; t++)
			{
				const int id = in.mux_thread_ids ? in.mux_thread_ids[t] : t;
				if(id < 0 || id > 1023)
					return fail(err, st, FXB_ERR_ARG, "bad VDIF thread id");
				for(int q : o.mux_tids)
					if(q == id)
						return fail(err, st, FXB_ERR_ARG, "duplicate VDIF thread id");
				o.mux_tids.push_back(id);
			}
		}
		job.stations.push_back(o);
	}
	for(int b = 0; b < d->nbaseline; b++)
	{
		const fxb_baseline &in = d->baselines[b];
		Job::Baseline o;
		o.ds1 = in.ds1;
		o.ds2 = in.ds2;
		if(in.ds1 < 0 || in.ds2 < 0 || in.ds1 >= d->nstation || in.ds2 >= d->nstation || in.ds1 == in.ds2)
			return fail(err, st, FXB_ERR_ARG, "baseline station index out of range");
		if(in.nprod < 1 || !in.prod_freq || !in.prod_band1 || !in.prod_band2)
			return fail(err, st, FXB_ERR_ARG, "baseline without products");
		o.prod_freq.assign(in.prod_freq, in.prod_freq + in.nprod);
		o.prod_b1.assign(in.prod_band1, in.prod_band1 + in.nprod);
		o.prod_b2.assign(in.prod_band2, in.prod_band2 + in.nprod);
		for(int p = 0; p < in.nprod; p++)
		{
			int f = o.prod_freq[p];
			if(f < 0 || f >= d->nfreq)
				return fail(err, st, FXB_ERR_ARG, "product frequency out of range");
			if(p > 0 && f != o.prod_freq[p - 1])
				for(int q = 0; q < p - 1; q++)
					if(o.prod_freq[q] == f)
						return fail(err, st, FXB_ERR_ARG, "products of one frequency must be contiguous");
			int b1 = o.prod_b1[p], b2 = o.prod_b2[p];
			const Job::Station &s1 = job.stations[o.ds1], &s2 = job.stations[o.ds2];
			if(b1 < 0 || b1 >= s1.nband + s1.nzoom() || b2 < 0 || b2 >= s2.nband + s2.nzoom())
				return fail(err, st, FXB_ERR_ARG, "product band index out of range");
			if(s1.total_freq(b1) != f || s2.total_freq(b2) != f)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "product bands must record the product frequency");
		}
		job.baselines.push_back(o);
	}
	job.subint_ns = d->subint_ns;
	job.fringe_rot_order = d->fringe_rot_order;
	job.write_autocorrs = d->write_autocorrs ? 1 : 0;
	job.xmac_kind = d->xmac_kind;
	job.inflight = std::max(1, std::min(8, d->max_subints_in_flight));

	// blockspersend (configuration.cpp:1852-1860); all stations must agree
	{
		const int S = (int)job.stations.size();
		double bps0 = -1.0;
		for(int s = 0; s < S; s++)
		{
			const fxb_freq &f = job.freqs[job.stations[s].band_freq[0]];
			double fftns = 2.0 * f.nchan * 1000.0 / (2.0 * f.bw_mhz);
			double bpsd = (double)d->subint_ns / fftns;
			int bps = (int)(bpsd + 0.5);
			if(std::fabs(bpsd - bps) > 1e-9 || bps < 1)
				return fail(err, st, FXB_ERR_ARG, "subint must hold a whole number of FFTs");
			if(bps0 >= 0 && bps != (int)bps0)
				return fail(err, st, FXB_ERR_UNSUPPORTED, "all stations must have the same FFTs per subint");
			bps0 = bps;
			job.blockspersend = bps;
			int64_t fsamp = (int64_t)job.stations[s].payload * 8 / (job.stations[s].nbits * job.stations[s].nband);
			double sps = 2e6 * f.bw_mhz;
			if(std::fabs(sps / fsamp - std::floor(sps / fsamp + 0.5)) > 1e-9)
				return fail(err, st, FXB_ERR_ARG, "whole frames per second required");
		}
	}

	// getMaxProducts (configuration.cpp:843-857)
	const int F = (int)job.freqs.size(), B = (int)job.baselines.size(), S = (int)job.stations.size();
	job.maxproducts = 0;
	for(auto &bl : job.baselines)
		for(int f = 0; f < F; f++)
		{
			int n = (int)std::count(bl.prod_freq.begin(), bl.prod_freq.end(), f);
			job.maxproducts = std::max(job.maxproducts, n);
		}
	job.bandsperautocorr = job.maxproducts > 2 ? 2 : 1;

	// frequency usage (configuration.cpp:325-368)
	job.freqused.assign(F, 0);
	job.equivused.assign(F, 0);
	for(auto &bl : job.baselines)
		for(int f : bl.prod_freq)
			job.freqused[f] = 1;
	for(int f = 0; f < F; f++)
	{
		if(job.freqused[f])
			continue;
		for(int k = 0; k < F; k++)
		{
			double bwdiff = job.freqs[f].bw_mhz - job.freqs[k].bw_mhz;
			double freqdiff = job.freqs[f].freq_mhz - job.freqs[k].freq_mhz;
			if(job.freqs[f].lower_sideband) freqdiff -= job.freqs[f].bw_mhz;
			if(job.freqs[k].lower_sideband) freqdiff += job.freqs[k].bw_mhz;
			if(bwdiff < 1e-9 && freqdiff < 1e-9 && job.freqs[f].nchan == job.freqs[k].nchan &&
			   job.freqs[f].chans_to_avg == job.freqs[k].chans_to_avg && job.freqused[k])
				job.equivused[f] = 1;
		}
	}

	// core-result layout
	int64_t idx = 0;
	job.bloff.assign((size_t)F * B, -1);
	job.bwoff.assign((size_t)F * B, -1);
	job.acoff.assign(S, 0);
	job.acwoff.assign(S, 0);
	auto nprod_f = [&](const Job::Baseline &bl, int f) {
		return (int)std::count(bl.prod_freq.begin(), bl.prod_freq.end(), f);
	};
	for(int f = 0; f < F; f++)
	{
		if(!job.freqused[f]) continue;
		for(int b = 0; b < B; b++)
		{
			int n = nprod_f(job.baselines[b], f);
			if(!n) continue;
			job.bloff[(size_t)f * B + b] = idx;
			idx += (int64_t)n * job.freqs[f].nchan / job.freqs[f].chans_to_avg;
		}
	}
	for(int f = 0; f < F; f++)
	{
		if(!job.freqused[f]) continue;
		for(int b = 0; b < B; b++)
		{
			int n = nprod_f(job.baselines[b], f);
			if(!n) continue;
			job.bwoff[(size_t)f * B + b] = idx;
			idx += n / 2 + n % 2;
		}
	}
	for(int s = 0; s < S; s++)
	{
		job.acoff[s] = idx;
		for(int bnd = 0; bnd < job.stations[s].nband + job.stations[s].nzoom(); bnd++)
		{
			int fi = job.stations[s].total_freq(bnd);
			if(job.freqused[fi] || job.equivused[fi])
				idx += (int64_t)job.bandsperautocorr * job.freqs[fi].nchan / job.freqs[fi].chans_to_avg;
		}
	}
	for(int s = 0; s < S; s++)
	{
		job.acwoff[s] = idx;
		int toadd = 0;
		for(int bnd = 0; bnd < job.stations[s].nband + job.stations[s].nzoom(); bnd++)
		{
			int fi = job.stations[s].total_freq(bnd);
			if(job.freqused[fi] || job.equivused[fi])
				toadd += job.bandsperautocorr;
		}
		toadd = (toadd + 1) / 2;
		if(toadd == 0) toadd = 1;
		idx += toadd;
	}
	// then each station's phase-cal tones, band by band (configuration.cpp:2423-2431)
	job.pcoff.assign(S, -1);
	for(int s = 0; s < S; s++)
	{
		const Job::Station &js = job.stations[s];
		if(!(js.pcal_interval > 0.0f))
			continue;
		job.pcoff[s] = idx;
		for(int bnd = 0; bnd < js.nband; bnd++)
		{
			Job::PcalBand pb;
			pb.station = s;
			pb.band = bnd;
			if(!pcal_band(job.freqs[js.band_freq[bnd]], js.pcal_interval, js.pcal_base, pb, err, st))
				return false;
			pb.core = idx;
			pb.bin_off = job.pcal_bins;
			job.pcal_bins += (pb.shift ? 2 : 1) * (int64_t)pb.nbins;
			idx += pb.ntones;
			job.pcal.push_back(pb);
		}
	}
	job.corelen = idx;

	// fractionalLoFreq (mode.cpp:89-105)
	job.fractionallofreq = false;
	for(auto &s : job.stations)
		for(int f : s.band_freq)
		{
			double lo = job.freqs[f].freq_mhz;
			if(std::fabs(lo - (int)(lo + 0.5)) > 0.000000001)
				job.fractionallofreq = true;
		}

	// rows per frequency, spectra and accumulator plans
	// (F-stage rows: recorded bands of frequencies with output, and recorded
	// bands that parent a zoom band with output; then the zoom bands of
	// frequencies with output, whose rows are gathered from their parents)
	auto fout = [&](int f) { return job.freqused[f] || job.equivused[f]; };
	const bool writecross = job.write_autocorrs && job.maxproducts > 2;
	job.rows.assign(F, {});
	job.band_row.assign(S, {});
	for(int s = 0; s < S; s++)
	{
		const Job::Station &js = job.stations[s];
		job.band_row[s].assign(js.nband + js.nzoom(), -1);
		std::vector<int> parent(js.nband, 0);
		for(int z = 0; z < js.nzoom(); z++)
			if(fout(js.zoom_freq[z]))
				parent[js.zoom_parent[z]] = 1;
		for(int bnd = 0; bnd < js.nband; bnd++)
		{
			int f = js.band_freq[bnd];
			if(!(fout(f) || parent[bnd]))
				continue;
			job.band_row[s][bnd] = (int)job.rows[f].size();
			job.rows[f].push_back({s, bnd});
		}
	}
	for(int s = 0; s < S; s++)
	{
		const Job::Station &js = job.stations[s];
		for(int z = 0; z < js.nzoom(); z++)
		{
			const int f = js.zoom_freq[z];
			for(int y = 0; y < z; y++)
				if(js.zoom_freq[y] == f && js.zoom_pol[y] == js.zoom_pol[z])
					return fail(err, st, FXB_ERR_ARG, "duplicate zoom band");
			if(!fout(f))
				continue;
			// a zoom band's cross-hand autocorrelation is its parent's
			// (mode.cpp:389-397): the station's first two zoom bands on this
			// frequency must then zoom the parent frequency's first two bands
			if(writecross)
			{
				const int pf = js.band_freq[js.zoom_parent[z]];
				std::vector<int> rec, zb;
				for(int b = 0; b < js.nband; b++)
					if(js.band_freq[b] == pf) rec.push_back(b);
				for(int y = 0; y < js.nzoom(); y++)
					if(js.zoom_freq[y] == f) zb.push_back(js.zoom_parent[y]);
				if(rec.size() >= 2)
				{
					std::vector<int> a(rec.begin(), rec.begin() + 2);
					std::sort(a.begin(), a.end());
					std::sort(zb.begin(), zb.end());
					if(zb != a)
						return fail(err, st, FXB_ERR_UNSUPPORTED,
						            "cross-hand autocorrelations need each zoom frequency in the parent's first two bands");
				}
			}
			job.band_row[s][js.nband + z] = (int)job.rows[f].size();
			job.rows[f].push_back({s, js.nband + z});
		}
	}
	job.plan.assign(F, {});
	const int T = job.blockspersend;
	std::vector<std::vector<int>> crossout(S);     // [s][band] -> cross-pol output index, -1
	for(int s = 0; s < S; s++)
	{
		crossout[s].assign(job.stations[s].nband + job.stations[s].nzoom(), -1);
	}
	int64_t spec = 0, acc = 0;
	for(int f = 0; f < F; f++)
	{
		Job::FreqPlan &pl = job.plan[f];
		pl.nrow = (int)job.rows[f].size();
		pl.nchan = job.freqs[f].nchan;
		if(pl.nrow == 0)
			continue;
		if(pl.nrow > 128)
			return fail(err, st, FXB_ERR_UNSUPPORTED, "more than 128 inputs on one frequency");
		pl.spec_off = spec;
		spec += (int64_t)T * pl.nrow * pl.nchan;
		pl.destA.assign((size_t)pl.nrow * pl.nrow, -1);
		pl.destB.assign((size_t)pl.nrow * pl.nrow, -1);
		pl.acc_off = acc;
		pl.xmac = fout(f);
		for(int r = 0; r < pl.nrow; r++)
		{
			const Job::Row &row = job.rows[f][r];
			const Job::Station &js = job.stations[row.station];
			if(row.band < js.nband)
				continue;
			const int z = row.band - js.nband, pb = js.zoom_parent[z];
			job.zooms.push_back({js.band_freq[pb], job.band_row[row.station][pb], f, r, js.zoom_choff[z], pl.nchan});
		}
		if(!pl.xmac)
			continue;
		int nout = 0;
		// baseline products, in core-result order
		for(int b = 0; b < B; b++)
		{
			const Job::Baseline &bl = job.baselines[b];
			int pf = 0;
			for(size_t p = 0; p < bl.prod_freq.size(); p++)
			{
				if(bl.prod_freq[p] != f) continue;
				int r1 = job.band_row[bl.ds1][bl.prod_b1[p]], r2 = job.band_row[bl.ds2][bl.prod_b2[p]];
				int o = nout++;
				if(r1 < r2)
				{
					if(pl.destA[(size_t)r1 * pl.nrow + r2] >= 0)
						return fail(err, st, FXB_ERR_UNSUPPORTED, "duplicate product");
					pl.destA[(size_t)r1 * pl.nrow + r2] = o;
				}
				else
				{
					if(pl.destB[(size_t)r2 * pl.nrow + r1] >= 0)
						return fail(err, st, FXB_ERR_UNSUPPORTED, "duplicate product");
					pl.destB[(size_t)r2 * pl.nrow + r1] = o;
				}
				job.outmap.push_back({acc + (int64_t)o * pl.nchan,
				                      job.bloff[(size_t)f * B + b] + (int64_t)pf * pl.nchan / job.freqs[f].chans_to_avg,
				                      pl.nchan, job.freqs[f].chans_to_avg, f, o});
				job.bweights.push_back({bl.ds1, bl.ds2, bl.prod_b1[p], bl.prod_b2[p], 2 * job.bwoff[(size_t)f * B + b] + pf});
				pf++;
			}
		}
		// autocorrelations: one output per row
		for(int r = 0; r < pl.nrow; r++)
			pl.destA[(size_t)r * pl.nrow + r] = nout++;
		// cross-pol autocorrelations (mode.cpp:1356-1369): the first two bands
		// of a station on this frequency; V[r0][r1] and its conjugate
		if(job.write_autocorrs)
			for(int s = 0; s < S; s++)
			{
				int idxs[2], cnt = 0;
				const Job::Station &js = job.stations[s];
				for(int bnd = 0; bnd < js.nband + js.nzoom() && cnt < 2; bnd++)
					if(js.total_freq(bnd) == f) idxs[cnt++] = bnd;
				if(cnt < 2) continue;
				int r0 = job.band_row[s][idxs[0]], r1 = job.band_row[s][idxs[1]];
				int o01 = nout++, o10 = nout++;
				// rows of one station are contiguous and ordered by band: r0 < r1
				pl.destA[(size_t)r0 * pl.nrow + r1] = o01;
				pl.destB[(size_t)r0 * pl.nrow + r1] = o10;
				crossout[s][idxs[0]] = o01;
				crossout[s][idxs[1]] = o10;
			}
		pl.nout = nout;
		acc += (int64_t)nout * pl.nchan;
	}
	job.spec_total = spec;
	job.acc_total = acc;

	// autocorrelation outputs and weights (core.cpp:1266-1363); a zoom band's
	// weight is its parent band's (core.cpp:1311-1322), which is the
	// station's FFT weight like every band's
	for(int s = 0; s < S; s++)
	{
		int64_t ridx = job.acoff[s];
		int64_t widx = 2 * job.acwoff[s];
		for(int pass = 0; pass < (writecross ? 2 : 1); pass++)
			for(int bnd = 0; bnd < job.stations[s].nband + job.stations[s].nzoom(); bnd++)
			{
				int f = job.stations[s].total_freq(bnd);
				if(!(job.freqused[f] || job.equivused[f])) continue;
				const Job::FreqPlan &pl = job.plan[f];
				int r = job.band_row[s][bnd];
				int64_t a;
				int o;
				if(pass == 0)
					o = pl.destA[(size_t)r * pl.nrow + r];
				else
					o = crossout[s][bnd];
				a = o >= 0 ? pl.acc_off + (int64_t)o * pl.nchan : -1;
				job.outmap.push_back({a, ridx, pl.nchan, job.freqs[f].chans_to_avg, f, o});
				ridx += pl.nchan / job.freqs[f].chans_to_avg;
				job.acweights.push_back({s, bnd, widx++});
			}
	}
	return true;
}

}  // namespace fxb
