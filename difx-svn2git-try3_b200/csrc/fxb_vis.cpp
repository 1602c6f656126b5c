// Integration output of the C ABI: amplitude calibration of an integrated
// core result (Visibility::writedata, mpifxcorr/src/visibility.cpp:348-620)
// and the SWIN ".difx" record writer (Visibility::writedifx and
// writeDiFXHeader, visibility.cpp:716-900, 1060-1140).
//
// The integration sum itself needs no code here: a context accumulates every
// subint it is given on the device until fxb_reset, which is what
// Visibility::addData (visibility.cpp:181-194) does with the core results
// sent to it.  Calibration is one pass over the integrated buffer per
// integration and runs on the host, in the reference's own arithmetic
// (float weights and scales, products formed in the order the reference
// writes them), so that the calibrated buffer and the records are
// bit-identical to the reference's for the same integrated core result.

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "fxb_internal.h"

namespace fxb {

namespace {

// Mode::getDecorrelationPercentage (mode.h:176, values mode.cpp:1594): the
// approximate correlation loss of 1..8-bit quantisation
const float kDecorrelation[8] = {0.63662f, 0.88f, 0.94f, 0.96f, 0.98f, 0.99f, 0.996f, 0.998f};

char opposite_pol(char p)
{
	if(p == 'R') return 'L';
	if(p == 'L') return 'R';
	if(p == 'X') return 'Y';
	if(p == 'Y') return 'X';
	return 'X';
}

// Per-integration constants (Visibility::changeConfig, visibility.cpp:1198-1200)
struct Integration {
	double meansubints, ffts;
};

Integration integration(const Job &job, const fxb_vis_params *p)
{
	Integration in;
	in.meansubints = p->int_time_s / (((double)job.subint_ns) / 1000000000.0);
	in.ffts = in.meansubints * job.blockspersend;
	return in;
}

bool used(const Job &job, int f) { return job.freqused[f] || job.equivused[f]; }

// distinct frequencies of a baseline in product order, with their products
struct BFreq {
	int f;
	std::vector<int> prods;   // indices into prod_*
};

std::vector<BFreq> baseline_freqs(const Job::Baseline &bl)
{
	std::vector<BFreq> out;
	for(size_t k = 0; k < bl.prod_freq.size(); k++)
	{
		const int f = bl.prod_freq[k];
		size_t j = 0;
		while(j < out.size() && out[j].f != f)
			j++;
		if(j == out.size())
			out.push_back({f, {}});
		out[j].prods.push_back((int)k);
	}
	return out;
}

// band of station s that records frequency f in the opposite polarisation of
// band k (Configuration::getDMatchingBand)
int matching_band(const Job &job, int s, int k)
{
	const Job::Station &st = job.stations[s];
	for(int b = 0; b < st.nband; b++)
		if(b != k && st.band_freq[b] == st.band_freq[k] && st.band_pol[b] != st.band_pol[k])
			return b;
	return k;
}

// autocorrelation weights [station][j][band] over the recorded and then the
// zoom bands (visibility.cpp:415-432)
std::vector<std::vector<std::vector<float>>> ac_weights(const Job &job, const Integration &in, const float *fr)
{
	const int S = (int)job.stations.size(), W = job.bandsperautocorr;
	std::vector<std::vector<std::vector<float>>> w(S);
	for(int i = 0; i < S; i++)
	{
		const Job::Station &st = job.stations[i];
		int64_t ri = job.acwoff[i] * 2;
		w[i].assign(W, std::vector<float>(st.total_bands(), 0.0f));
		for(int j = 0; j < W; j++)
			for(int k = 0; k < st.total_bands(); k++)
				if(used(job, st.total_freq(k)))
					w[i][j][k] = fr[ri++] / in.ffts;
	}
	return w;
}

// A zoom band carries a fraction of its parent's samples: the visibility
// normalisation multiplies by zoom / parent bandwidth in float
// (visibility.cpp:486-499, 560-566); 1 for a recorded band.
float zoom_modifier(const Job &job, int s, int k)
{
	const Job::Station &st = job.stations[s];
	if(k < st.nband)
		return 1.0f;
	float m = 1.0f;
	m = (float)(m * job.freqs[st.total_freq(k)].bw_mhz);
	m = (float)(m / job.freqs[st.band_freq[st.zoom_parent[k - st.nband]]].bw_mhz);
	return m;
}

float baseline_weight(const Job &job, const Integration &in, const float *fr, int b, int f, int pp)
{
	const size_t B = job.baselines.size();
	return fr[job.bwoff[(size_t)f * B + b] * 2 + pp] / in.ffts;
}

}  // namespace

static fxb_status calibrate(const Job &job, const fxb_vis_params *p, float *fr)
{
	const Integration in = integration(job, p);
	const int S = (int)job.stations.size(), B = (int)job.baselines.size(), W = job.bandsperautocorr;
	auto tsys = [&](int s) { return p->tsys ? p->tsys[s] : 0.0; };
	// The reference looks up the opposite-hand band of a zoom band with the
	// band's index into the zoom band tables (Configuration::getDMatchingBand,
	// configuration.cpp:907-922), which reads past them: Tsys scaling of the
	// cross-hand autocorrelations of zoom bands has no defined result there.
	if(job.write_autocorrs && W == 2)
		for(int i = 0; i < S; i++)
			if(tsys(i) > 0.0)
				for(int k = job.stations[i].nband; k < job.stations[i].total_bands(); k++)
					if(used(job, job.stations[i].total_freq(k)))
						return FXB_ERR_UNSUPPORTED;
	const auto acw = ac_weights(job, in, fr);

	// band averages of the (parallel-hand) autocorrelations, for Tsys scaling
	// (visibility.cpp:446-464; genericMean_32fc: float sum, then / length)
	std::vector<std::vector<float>> accal(S);
	for(int i = 0; i < S; i++)
	{
		accal[i].assign(job.stations[i].total_bands(), 0.0f);
		if(tsys(i) > 0.0)
		{
			int64_t ri = job.acoff[i];
			for(int k = 0; k < job.stations[i].total_bands(); k++)
			{
				const int f = job.stations[i].total_freq(k);
				if(!used(job, f))
					continue;
				const int fc = job.freqs[f].nchan / job.freqs[f].chans_to_avg;
				float re = 0.0f;
				for(int c = 0; c < fc; c++)
					re += fr[2 * (ri + c)];
				if(fc > 0)
					re /= fc;
				accal[i][k] = re;
				ri += fc;
			}
		}
	}

	// cross correlations (visibility.cpp:466-545)
	for(int b = 0; b < B; b++)
	{
		const Job::Baseline &bl = job.baselines[b];
		const int ds1 = bl.ds1, ds2 = bl.ds2;
		for(const BFreq &bf : baseline_freqs(bl))
		{
			const int f = bf.f;
			int64_t ri = job.bloff[(size_t)f * B + b];
			const int fc = job.freqs[f].nchan / job.freqs[f].chans_to_avg;
			for(size_t k = 0; k < bf.prods.size(); k++)
			{
				const int b1 = bl.prod_b1[bf.prods[k]], b2 = bl.prod_b2[bf.prods[k]];
				const float bw = baseline_weight(job, in, fr, b, f, (int)k);
				float scale;
				if(tsys(ds1) > 0.0 && tsys(ds2) > 0.0)
				{
					const float divisor = kDecorrelation[job.stations[ds1].nbits - 1] *
					                      kDecorrelation[job.stations[ds2].nbits - 1] * accal[ds1][b1] * accal[ds2][b2] /
					                      (acw[ds1][0][b1] * acw[ds2][0][b2]);
					if(divisor > 0.0f && bw > 0)
						scale = (float)(std::sqrt(tsys(ds1) * tsys(ds2) / divisor) / bw);
					else
						scale = 0.0f;
				}
				else if(bw > 0.0f)
				{
					scale = (float)(1.0 / (bw * in.meansubints *
					                       ((float)(job.blockspersend * 2 * fc * job.freqs[f].chans_to_avg))));
					if(b1 >= job.stations[ds1].nband)
						scale *= std::sqrt(zoom_modifier(job, ds1, b1));
					if(b2 >= job.stations[ds2].nband)
						scale *= std::sqrt(zoom_modifier(job, ds2, b2));
				}
				else
					scale = 0.0f;
				if(scale > 0.0f)
					for(int c = 0; c < 2 * fc; c++)
						fr[2 * ri + c] *= scale;
				ri += fc;
			}
		}
	}

	// autocorrelations (visibility.cpp:547-595)
	if(job.write_autocorrs)
	{
		for(int i = 0; i < S; i++)
		{
			int64_t ri = job.acoff[i] * 2;
			for(int j = 0; j < W; j++)
				for(int k = 0; k < job.stations[i].total_bands(); k++)
				{
					const int f = job.stations[i].total_freq(k);
					if(!used(job, f))
						continue;
					const int fc = job.freqs[f].nchan / job.freqs[f].chans_to_avg;
					float scale = 0.0f;
					if(tsys(i) > 0.0)
					{
						const float divisor = std::sqrt(accal[i][k] * accal[i][j == 0 ? k : matching_band(job, i, k)]);
						if(divisor > 0.0f)
							scale = (float)(tsys(i) / divisor);
					}
					else if(acw[i][j][k] > 0.0f)
					{
						scale = (float)(1.0 / (acw[i][j][k] * in.meansubints *
						                       ((float)(job.blockspersend * 2 * fc * job.freqs[f].chans_to_avg))));
						if(k >= job.stations[i].nband)
							scale *= zoom_modifier(job, i, k);
					}
					if(scale > 0.0f)
						for(int c = 0; c < 2 * fc; c++)
							fr[ri + c] *= scale;
					ri += 2 * fc;
				}
		}
	}

	// phase-cal tones, recorded band by recorded band (visibility.cpp:586-609):
	// normalised by the band's autocorrelation weight, or by the data alone
	// when zoom bands leave the recorded band without one
	for(const Job::PcalBand &pb : job.pcal)
	{
		const int i = pb.station, j = pb.band;
		const fxb_freq &f = job.freqs[job.stations[i].band_freq[j]];
		const int fc = f.nchan / f.chans_to_avg;
		double a = acw[i][0][j];
		if(a == 0.0 && job.stations[i].total_bands() > job.stations[i].nband)
			a = 1.0;
		if(a > 0.0)
		{
			const float scale = (float)(1.0 / (a * in.meansubints * ((float)(job.blockspersend * 2 * fc * f.chans_to_avg))));
			for(int c = 0; c < 2 * pb.ntones; c++)
				fr[2 * pb.core + c] *= scale;
		}
	}
	return FXB_OK;
}

namespace {

void put(std::vector<char> &o, const void *p, size_t n)
{
	const char *c = (const char *)p;
	o.insert(o.end(), c, c + n);
}

// one SWIN record header (Visibility::writeDiFXHeader, visibility.cpp:1100-1135):
// sync word, header version, baseline number, MJD, seconds, configuration,
// source, frequency, polarisation pair, pulsar bin, weight, u, v, w
void header(std::vector<char> &o, int bnum, int mjd, double sec, int cfg, int src, int freq, char p0, char p1,
            int bin, float weight, const double *uvw)
{
	const uint32_t sync = 0xFF00FF00u;
	const int32_t version = 1;
	const int32_t v[4] = {version, bnum, mjd, 0};
	put(o, &sync, 4);
	put(o, v, 12);
	put(o, &sec, 8);
	const int32_t w[3] = {cfg, src, freq};
	put(o, w, 12);
	o.push_back(p0);
	o.push_back(p1);
	put(o, &bin, 4);
	const double dw = weight;
	put(o, &dw, 8);
	put(o, uvw, 24);
}

}  // namespace

static fxb_status swin_write(const Job &job, const fxb_vis_params *p, const float *fr, const char *dir,
                             std::string &err)
{
	const Integration in = integration(job, p);
	const int S = (int)job.stations.size(), B = (int)job.baselines.size(), W = job.bandsperautocorr;
	auto tel = [&](int s) { return p->telescope ? p->telescope[s] : s; };
	const int isec = p->start_sec + p->scan_start_sec + p->int_start_sec;
	const int mjd = p->start_mjd + isec / 86400;
	const double sec = double(isec % 86400) + ((double)p->int_start_ns) / 1000000000.0 + p->int_time_s / 2.0;
	const double zero[3] = {0.0, 0.0, 0.0};
	std::vector<char> o;

	// baselines: frequency by frequency, product by product, weight > 0 only
	for(int b = 0; b < B; b++)
	{
		const Job::Baseline &bl = job.baselines[b];
		const int bnum = (tel(bl.ds1) + 1) * 256 + (tel(bl.ds2) + 1);
		const double *uvw = p->uvw ? p->uvw + 3 * b : zero;
		for(const BFreq &bf : baseline_freqs(bl))
		{
			const int f = bf.f;
			int64_t ri = job.bloff[(size_t)f * B + b];
			const int fc = job.freqs[f].nchan / job.freqs[f].chans_to_avg;
			for(size_t k = 0; k < bf.prods.size(); k++)
			{
				const float bw = baseline_weight(job, in, fr, b, f, (int)k);
				if(bw > 0.0f)
				{
					const int b1 = bl.prod_b1[bf.prods[k]], b2 = bl.prod_b2[bf.prods[k]];
					header(o, bnum, mjd, sec, p->config_index, p->source_index, f, job.stations[bl.ds1].total_pol(b1),
					       job.stations[bl.ds2].total_pol(b2), 0, bw, uvw);
					put(o, fr + 2 * ri, sizeof(float) * 2 * fc);
				}
				ri += fc;
			}
		}
	}
	// autocorrelations (visibility.cpp:834-880), after the baselines
	if(job.write_autocorrs)
	{
		const auto acw = ac_weights(job, in, fr);
		for(int i = 0; i < S; i++)
		{
			const int bnum = 257 * (tel(i) + 1);
			int64_t ri = job.acoff[i];
			for(int j = 0; j < W; j++)
				for(int k = 0; k < job.stations[i].total_bands(); k++)
				{
					const int f = job.stations[i].total_freq(k);
					if(!used(job, f))
						continue;
					const int fc = job.freqs[f].nchan / job.freqs[f].chans_to_avg;
					if(acw[i][j][k] > 0.0f)
					{
						const char p0 = job.stations[i].total_pol(k);
						header(o, bnum, mjd, sec, p->config_index, p->source_index, f, p0, j == 0 ? p0 : opposite_pol(p0),
						       0, acw[i][j][k], zero);
						put(o, fr + 2 * ri, sizeof(float) * 2 * fc);
					}
					ri += fc;
				}
		}
	}
	char name[64];
	snprintf(name, sizeof(name), "/DIFX_%05d_%06d.s%04d.b%04d", p->start_mjd, p->start_sec, 0, 0);
	const std::string path = std::string(dir) + name;
	FILE *fp = fopen(path.c_str(), "ab");
	if(!fp)
	{
		err = "cannot open " + path;
		return FXB_ERR_ARG;
	}
	const size_t n = fwrite(o.data(), 1, o.size(), fp);
	const bool ok = fclose(fp) == 0 && n == o.size();
	if(!ok)
	{
		err = "short write to " + path;
		return FXB_ERR_DATA;
	}
	return FXB_OK;
}

// One line per station and integration of its calibrated phase-cal tones,
// appended to PCAL_<mjd>_<sec>_<station>, which starts with the reference's
// comment header (Visibility::initialisePcalFiles, visibility.cpp:104-135;
// the line: Visibility::writedifx, visibility.cpp:928-990).
static fxb_status pcal_write(const Job &job, const fxb_vis_params *p, const float *fr, const char *dir,
                             std::string &err)
{
	const int S = (int)job.stations.size();
	const int isec = p->start_sec + p->scan_start_sec + p->int_start_sec;
	const int dumpmjd = p->start_mjd + isec / 86400;
	const double dumpseconds = double(isec % 86400) + ((double)p->int_start_ns) / 1000000000.0 + p->int_time_s / 2.0;
	const double pcalmjd = dumpmjd + dumpseconds / 86400.0;
	for(int i = 0; i < S; i++)
	{
		const Job::Station &st = job.stations[i];
		if(!(st.pcal_interval > 0.0f))
			continue;
		char nm[32];
		snprintf(nm, sizeof(nm), "DS%d", i);
		const std::string name = p->names && p->names[i] ? p->names[i] : nm;
		std::vector<const Job::PcalBand *> bands;
		int maxtones = 0;
		for(const Job::PcalBand &pb : job.pcal)
			if(pb.station == i)
			{
				bands.push_back(&pb);
				maxtones = std::max(maxtones, pb.ntones);
			}
		char buf[256];
		snprintf(buf, sizeof(buf), "%s %13.7f %9.7f %d %d %d", name.c_str(), pcalmjd, p->int_time_s / 86400.0, i,
		         st.nband, maxtones);
		std::string line = buf;
		bool nonzero = false;
		for(const Job::PcalBand *pb : bands)
		{
			for(int t = 0; t < maxtones; t++)
			{
				if(t >= pb->ntones)
				{
					line += " -1 0 0 0";
					continue;
				}
				// tone frequencies (configuration.cpp:1799-1801, 1830-1833); a band
				// without a tone has one at 0
				double hz = 0.0;
				if(pb->nbins > 0 || pb->tonefreq != 0.0)
					hz = pb->lsb ? 1e6 * pb->tonefreq - double(t) * 1e6 * st.pcal_interval - 1e6 * st.pcal_base
					             : 1e6 * pb->tonefreq + t * 1e6 * st.pcal_interval + 1e6 * st.pcal_base;
				const double tonefreq = 1e-6 * hz;
				const float re = fr[2 * (pb->core + t)], im = fr[2 * (pb->core + t) + 1];
				snprintf(buf, sizeof(buf), " %.12g %c %12.5e %12.5e", tonefreq, st.band_pol[pb->band], re,
				         pb->lsb ? im : -im);
				if(re != 0.0 && -im != 0.0)
					nonzero = true;
				line += buf;
			}
		}
		if(!nonzero)
			continue;
		char fname[64];
		snprintf(fname, sizeof(fname), "/PCAL_%05d_%06d_", p->start_mjd, p->start_sec);
		const std::string path = std::string(dir) + fname + name;
		FILE *fp = fopen(path.c_str(), "r");
		const bool exists = fp != nullptr;
		if(fp)
			fclose(fp);
		fp = fopen(path.c_str(), "a");
		if(!fp)
		{
			err = "cannot open " + path;
			return FXB_ERR_ARG;
		}
		bool ok = true;
		if(!exists)
			ok = fprintf(fp, "# DiFX-derived pulse cal data\n# File version = 1\n# Start MJD = %d\n"
			                 "# Start seconds = %d\n# Telescope name = %s\n",
			             p->start_mjd, p->start_sec, name.c_str()) > 0;
		ok = ok && fprintf(fp, "%s\n", line.c_str()) > 0;
		ok = (fclose(fp) == 0) && ok;
		if(!ok)
		{
			err = "short write to " + path;
			return FXB_ERR_DATA;
		}
	}
	return FXB_OK;
}

fxb_status vis_pcal_write(const Job &job, const fxb_vis_params *p, const float *coreresult, const char *dir,
                          std::string &err)
{
	if(!p || !coreresult || !dir || p->int_time_s <= 0.0)
		return FXB_ERR_ARG;
	return pcal_write(job, p, coreresult, dir, err);
}

fxb_status vis_calibrate(const Job &job, const fxb_vis_params *p, float *coreresult)
{
	if(!p || !coreresult || p->int_time_s <= 0.0)
		return FXB_ERR_ARG;
	return calibrate(job, p, coreresult);
}

fxb_status vis_swin_write(const Job &job, const fxb_vis_params *p, const float *coreresult, const char *dir,
                          std::string &err)
{
	if(!p || !coreresult || !dir || p->int_time_s <= 0.0)
		return FXB_ERR_ARG;
	return swin_write(job, p, coreresult, dir, err);
}

}  // namespace fxb
