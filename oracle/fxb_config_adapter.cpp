/* Configuration -> fxb_job_desc and Model -> per-subint delay interpolators
 * (see fxb_config_adapter.h).  Compiled against the reference's headers. */
#include <cmath>
#include <limits>

#include "fxb_config_adapter.h"
#include "mode.h"
#include "model.h"

namespace {

/* The per-frequency corrections and the fringe-rotation order reach a
 * datastream only through its Mode (getMode passes the datastream table's
 * arrays to the constructor, configuration.cpp:1009); a class derived from
 * Mode may name its protected members, and the member pointers so formed
 * read them from any Mode. */
struct ModeFields : Mode
{
	static const double *clock(const Mode *m) { return m->*(&ModeFields::recordedfreqclockoffsets); }
	static const double *delta(const Mode *m) { return m->*(&ModeFields::recordedfreqclockoffsetsdelta); }
	static const double *phase(const Mode *m) { return m->*(&ModeFields::recordedfreqphaseoffset); }
	static const double *looff(const Mode *m) { return m->*(&ModeFields::recordedfreqlooffsets); }
	static int order(const Mode *m) { return m->*(&ModeFields::fringerotationorder); }
	static int dsb(const Mode *m) { return m->*(&ModeFields::usedouble); }
	static u8 *&workbuf(Mode *m) { return m->*(&ModeFields::fftbuffer); }
};

}  // namespace

void fxb_delete_mode(Mode *m)
{
#if defined(ARCH) && defined(GENERIC) && (ARCH == GENERIC)
	if(m && ModeFields::order(m) == 0)
		ModeFields::workbuf(m) = 0;
#endif
	delete m;
}

namespace {

void delete_mode(Mode *m, int)
{
	fxb_delete_mode(m);
}

}  // namespace

bool fxb_desc_from_configuration(Configuration *c, int ci, int32_t xmac_kind, FxbConfigDesc &d, std::string &err)
{
	d = FxbConfigDesc();
	const int nfreq = c->getFreqTableLength();
	for(int f = 0; f < nfreq; f++)
	{
		fxb_freq q;
		q.freq_mhz = c->getFreqTableFreq(f);
		q.bw_mhz = c->getFreqTableBandwidth(f);
		q.nchan = c->getFNumChannels(f);
		q.lower_sideband = c->getFreqTableLowerSideband(f) ? 1 : 0;
		q.chans_to_avg = c->getFChannelsToAverage(f);
		q.reserved = 0;
		d.freqs.push_back(q);
	}
	const int nds = c->getNumDataStreams();
	int order = 1;
	// every array is sized before any pointer into it is taken
	d.ints.reserve(3 * nds + 3 * c->getNumBaselines());
	d.pols.reserve(2 * nds);
	d.corr.reserve(4 * nds);
	for(int ds = 0; ds < nds; ds++)
	{
		fxb_station s = fxb_station();
		const Configuration::dataformat fmt = c->getDataFormat(ci, ds);
		if(fmt != Configuration::VDIF && fmt != Configuration::VDIFL && fmt != Configuration::INTERLACEDVDIF)
		{
			err = "datastream " + std::to_string(ds) + " is not VDIF";
			return false;
		}
		s.complex_sampling = c->getDSampling(ci, ds) == Configuration::COMPLEX ? 1 : 0;
		const int header = fmt == Configuration::VDIFL ? 16 : 32;
		s.nbits = c->getDNumBits(ci, ds);
		s.header_bytes = header;
		s.payload_bytes = c->getFrameBytes(ci, ds) - header;
		if(fmt == Configuration::INTERLACEDVDIF)
		{
			// the Mode reads the muxer's frames: one thread's payload per band
			// thread (configuration.cpp:1001-1008)
			s.mux_threads = c->getDNumMuxThreads(ci, ds);
			s.payload_bytes *= s.mux_threads;
		}
		s.nband = c->getDNumRecordedBands(ci, ds);
		s.nzoom = c->getDNumZoomBands(ci, ds);
		std::vector<int32_t> bf(s.nband), zf(s.nzoom > 0 ? s.nzoom : 1);
		std::vector<char> bp(s.nband + 1, 0), zp((s.nzoom > 0 ? s.nzoom : 1) + 1, 0);
		for(int b = 0; b < s.nband; b++)
		{
			bf[b] = c->getDRecordedFreqIndex(ci, ds, b);
			bp[b] = c->getDRecordedBandPol(ci, ds, b);
		}
		for(int z = 0; z < s.nzoom; z++)
		{
			zf[z] = c->getDZoomFreqIndex(ci, ds, z);
			zp[z] = c->getDZoomBandPol(ci, ds, z);
		}
		d.ints.push_back(bf);
		s.band_freq = d.ints.back().data();
		d.ints.push_back(zf);
		s.zoom_freq = d.ints.back().data();
		d.pols.push_back(bp);
		s.band_pol = d.pols.back().data();
		d.pols.push_back(zp);
		s.zoom_pol = d.pols.back().data();
		s.pcal_interval_mhz = c->getDPhaseCalIntervalMHz(ci, ds);
		s.pcal_base_mhz = c->getDPhaseCalBaseMHz(ci, ds);
		// per-frequency corrections, per band of the frequency
		Mode *m = c->getMode(ci, ds);
		if(!m || !m->initialisedOK())
		{
			delete_mode(m, m ? ModeFields::order(m) : 1);
			err = "no Mode for datastream " + std::to_string(ds);
			return false;
		}
		order = ModeFields::order(m);
		if(s.complex_sampling && ModeFields::dsb(m))
		{
			delete_mode(m, order);
			err = "datastream " + std::to_string(ds) + " is complex double-sideband sampled";
			return false;
		}
		const double *src[4] = {ModeFields::clock(m), ModeFields::delta(m), ModeFields::phase(m), ModeFields::looff(m)};
		const double **dst[4] = {&s.band_clock_us, &s.band_clock_delta_us, &s.band_phase_deg, &s.band_lo_offset_hz};
		for(int q = 0; q < 4; q++)
		{
			std::vector<double> v(s.nband);
			for(int b = 0; b < s.nband; b++)
				v[b] = src[q][c->getDLocalRecordedFreqIndex(ci, ds, b)];
			d.corr.push_back(v);
			*dst[q] = d.corr.back().data();
		}
		delete_mode(m, order);
		d.stations.push_back(s);
	}
	const int nbl = c->getNumBaselines();
	for(int b = 0; b < nbl; b++)
	{
		fxb_baseline bl = fxb_baseline();
		bl.ds1 = c->getBOrderedDataStream1Index(ci, b);
		bl.ds2 = c->getBOrderedDataStream2Index(ci, b);
		std::vector<int32_t> pf, p1, p2;
		for(int lf = 0; lf < c->getBNumFreqs(ci, b); lf++)
			for(int p = 0; p < c->getBNumPolProducts(ci, b, lf); p++)
			{
				pf.push_back(c->getBFreqIndex(ci, b, lf));
				p1.push_back(c->getBDataStream1BandIndex(ci, b, lf, p));
				p2.push_back(c->getBDataStream2BandIndex(ci, b, lf, p));
			}
		bl.nprod = (int32_t)pf.size();
		d.ints.push_back(pf);
		bl.prod_freq = d.ints.back().data();
		d.ints.push_back(p1);
		bl.prod_band1 = d.ints.back().data();
		d.ints.push_back(p2);
		bl.prod_band2 = d.ints.back().data();
		d.baselines.push_back(bl);
	}
	d.desc.nfreq = nfreq;
	d.desc.freqs = d.freqs.data();
	d.desc.nstation = nds;
	d.desc.stations = d.stations.data();
	d.desc.nbaseline = nbl;
	d.desc.baselines = d.baselines.data();
	d.desc.subint_ns = c->getSubintNS(ci);
	d.desc.fringe_rot_order = order;
	d.desc.write_autocorrs = c->writeAutoCorrs(ci) ? 1 : 0;
	d.desc.xmac_kind = xmac_kind;
	d.desc.max_subints_in_flight = 2;
	return true;
}

int fxb_interpolators_from_model(Configuration *c, int ci, int scan, int sec, int ns, double *interp)
{
	Model *model = c->getModel();
	const int srcindex = model->getNumPhaseCentres(scan) == 1 ? 1 : 0;
	const int bps = c->getBlocksPerSend(ci);
	int missing = 0;
	for(int ds = 0; ds < c->getNumDataStreams(); ds++)
	{
		const int nchan = c->getFNumChannels(c->getDRecordedFreqIndex(ci, ds, 0));
		const double sampletime = 1.0 / (2.0 * c->getDRecordedBandwidth(ci, ds, 0));   // us
		const double timespan = bps * 2 * nchan * sampletime / 1e6;
		double *k = interp + 3 * ds;
		const bool ok = model->calculateDelayInterpolator(scan, (double)sec + ns / 1e9, timespan, bps,
		                                                  c->getDModelFileIndex(ci, ds), srcindex, 2, k);
		const int intclockseconds = int(floor(c->getDClockCoeff(ci, ds, 0) / 1000000.0 + 0.5));
		k[2] -= 1000000 * intclockseconds;
		if(!ok)
		{
			k[0] = k[1] = k[2] = std::numeric_limits<double>::quiet_NaN();
			missing++;
		}
	}
	return missing;
}
