// Internal structures shared by the host runtime and the sm_100a kernels.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fxb200.h"

namespace fxb {

constexpr int kFlagsPerInt = 30;          // mpifxcorr/src/mpifxcorr.h:39
constexpr int kMaxStations = 64;
constexpr int kMaxBandsPerStation = 64;
constexpr int kMaxPolyOrder = 5;          // MAX_POLY_ORDER of the .im reader
constexpr int kMaxPolys = 64;
constexpr int kTile = 4;                  // rows per register tile in the FP32 XMAC

// FFT status codes written by the delay kernel (why Mode::process zeroes an FFT).
enum FftStatus : int32_t {
	kFftZero = 0,        // flagged invalid, out of range, or zero weight
	kFftOk = 1
};

// Per (station, FFT) parameters derived in FP64 by the delay kernel
// (Mode::process, mode.cpp:671-840, and Mk5Mode::unpack, mk5mode.cpp:104-177).
struct FftParam {
	int32_t status;
	int32_t nearest;      // nearest sample, relative to the start of the station buffer
	int32_t stuck;        // samples [stuck, N) of the window decode to zero (8-bit 2/4-channel blanking)
	float weight;         // Mode::getDataWeight
	float fse;            // fractional sample error (us), float as in mode.cpp:772
	uint32_t fmask;       // validity of the frames of the window [nearest, nearest + N): bit k = frame nearest/fs + k
	double averagedelay;  // us
	double a, b, c;       // fringe-rotation coefficients of the order in use
	int32_t integerdelay;
	int32_t mflags;       // 1: fmask covers every frame of the window (at most 32 frames)
};

// Station description on the device.
struct DevStation {
	int32_t nbits, payload, header, nband;
	int32_t framebytes;
	int32_t framesamples;
	int32_t gran;           // samplegranularity
	int32_t nchan;          // channels per band (common to all bands of a station)
	int32_t fftchannels;    // 2*nchan
	int32_t asl;            // array stride length (calcstridelength(nchan))
	int32_t sticky;         // 8-bit 2/4-channel blank semantics
	int32_t mux;            // INTERLACEDVDIF: per-band weights, EDV4 band blanking
	int32_t bpbn, bpbd;     // bytes-per-block numerator/denominator of Mode
	// raw INTERLACEDVDIF reads (muxraw): the threads' frames, one band each;
	// the geometry above is the muxed stream's
	int32_t muxraw, nthr, inframebytes, fps;
	int32_t cplx;           // complex sampling: nchan-point complex FFT, real and imaginary fields per sample
	int32_t pad_;
	int32_t tmap[32];       // VDIF thread id of each band's thread
	double bw;              // MHz
	double sampletime;      // us
	int32_t npoly, order, interval;
	double poly0;
	double coeffs[kMaxPolys * (kMaxPolyOrder + 1)];
};

// One band of one station as the F kernel sees it.
struct DevBand {
	int32_t freq;           // frequency-table index
	int32_t row;            // row of this band within its frequency's spectra
	int32_t lsb;
	int32_t pad;
	double lofreq;          // MHz
};

// Per-subint inputs of one station.
struct DevSubintStation {
	const uint8_t *buf;
	int64_t nbytes;
	int32_t datasec, datans;
	int32_t invalid_subint; // no delay model for this time (subint torched)
	int32_t subsec, subns;  // subint start (the setOffsets time), the same for every station
	int32_t interp_given;   // interp was given by the caller (no device evaluation of the polynomials)
	double interp[3];       // quadratic delay interpolator (Mode::setOffsets)
	// raw INTERLACEDVDIF reads: buf holds nin thread frames; the device
	// places them into frame slots ([nslot][nthr] input frame or -1), writes
	// the muxed stream's headers (16 words per output frame: header, first
	// and last 64-bit payload words) and then sets nbytes / datasec / datans
	// to the muxed stream's and k0 to its first slot
	int32_t *mux_slot;
	uint32_t *mux_hdr;
	int32_t *mux_status;    // [0] error, [2] first filled slot
	int32_t mux_nin, mux_nproc, mux_nslot, mux_k0;
};

// Host-side job after validation.
struct Job {
	std::vector<fxb_freq> freqs;
	struct Station {
		int nbits, payload, header, nband;
		std::vector<int> band_freq;
		std::vector<char> band_pol;
		// zoom bands: frequency, polarisation, parent recorded band and the
		// parent channel of the zoom band's first channel
		std::vector<int> zoom_freq, zoom_parent, zoom_choff;
		std::vector<char> zoom_pol;
		int nzoom() const { return (int)zoom_freq.size(); }
		float pcal_interval = 0.0f, pcal_base = 0.0f;   // phase-cal comb (MHz), float as the reference
		int mux_threads = 0;                           // INTERLACEDVDIF: per-band data weights
		bool mux_raw = false;                          // buffers are raw reads, de-interleaved in the F stage
		bool cplx = false;                             // complex (single-sideband) sampling
		std::vector<int> mux_tids;                     // raw reads: VDIF thread id of each band's thread
		// per band, of its recorded frequency: clock offset and R/L delta (us),
		// phase offset (degrees), LO offset (Hz); has_corr: any of them nonzero
		std::vector<double> clk, dclk, phase, looff;
		bool has_corr = false;
		// frequency of band k: recorded bands, then zoom bands
		int total_freq(int k) const { return k < nband ? band_freq[k] : zoom_freq[k - nband]; }
		char total_pol(int k) const { return k < nband ? band_pol[k] : zoom_pol[k - nband]; }
		int total_bands() const { return nband + nzoom(); }
		int npoly = 0, order = 0, interval = 0;
		double poly0 = 0.0;
		std::vector<double> coeffs;
	};
	std::vector<Station> stations;
	struct Baseline {
		int ds1, ds2;
		std::vector<int> prod_freq, prod_b1, prod_b2;
	};
	std::vector<Baseline> baselines;
	int64_t subint_ns = 0;
	int fringe_rot_order = 1;
	int write_autocorrs = 1;
	int xmac_kind = 0;
	int inflight = 2;

	// derived
	int blockspersend = 0;
	int maxproducts = 0;
	int bandsperautocorr = 1;
	bool fractionallofreq = false;
	std::vector<int> freqused, equivused;
	int64_t corelen = 0;
	std::vector<int64_t> bloff, bwoff, acoff, acwoff;   // core-result offsets (complex index)

	// rows of every used frequency: (station, band) in station order
	struct Row { int station, band; };
	std::vector<std::vector<Row>> rows;                  // [freq]
	std::vector<std::vector<int>> band_row;              // [station][band, then zoom band] -> row in its freq
	// XMAC outputs per frequency: accumulator offsets
	struct FreqPlan {
		int nrow = 0;
		int nchan = 0;
		int64_t spec_off = 0;      // offset (complex) of this freq's spectra [T][nrow][nchan]
		int64_t acc_off = 0;       // offset (complex) of this freq's accumulators [nout][nchan]
		int nout = 0;
		std::vector<int> destA;    // [nrow*nrow] output index of V[i][j] (i<=j) or -1
		std::vector<int> destB;    // [nrow*nrow] output index receiving conj(V[i][j]) or -1
		bool xmac = false;         // false: spectra only (parents of zoom bands), no XMAC
	};
	std::vector<FreqPlan> plan;                           // [freq]
	int64_t spec_total = 0;       // complex values of spectra for one subint
	int64_t acc_total = 0;        // complex accumulators
	// output descriptors for finalisation
	struct OutMap {
		int64_t acc;     // accumulator offset (complex) of the first channel, [out][chan] layout
		int64_t core;    // core-result offset (complex) of the first output channel
		int nchan, avg;
		int freq, out;   // frequency and output index within it (out < 0: no accumulator)
	};
	std::vector<OutMap> outmap;
	// zoom bands: spectra rows gathered from the parent band's spectra
	struct ZoomCopy { int src_freq, src_row, dst_freq, dst_row, choff, nchan; };
	std::vector<ZoomCopy> zooms;
	// phase cal: per recorded band of a station with extraction, the tones,
	// the bins the samples are folded into (0: no tone in the band, one zero
	// tone), the DFT bin of the first tone and the bin step between tones
	struct PcalBand {
		int station, band, ntones, nbins, first, step;
		int shift;          // shifting extractor: samples rotated by this offset (Hz) into complex bins; else 0
		double tonefreq;    // comb tone nearest the LO inside the band, before the base (MHz); 0: no tone
		int lsb;
		int64_t fs;         // samples per second
		int64_t core;       // core-result offset (complex) of the band's first tone
		int64_t bin_off;    // offset (doubles) of the band's bins in the bin accumulator (complex bins: 2 per bin)
	};
	std::vector<PcalBand> pcal;
	int64_t pcal_bins = 0;
	std::vector<int64_t> pcoff;   // core-result offset of each station's tones, -1 without phase cal
	// weight plans
	// band indices pick the per-band data weights of INTERLACEDVDIF stations
	struct BWeight { int s1, s2, b1, b2; int64_t dst_float; };
	std::vector<BWeight> bweights;
	// both autocorrelation passes carry the band's own weight (Core writes
	// Mode::getWeight(false, band) for each, core.cpp:1324-1357)
	struct ACWeight { int s; int band; int64_t dst_float; };
	std::vector<ACWeight> acweights;
};

bool build_job(const fxb_job_desc *d, Job &job, std::string &err, fxb_status &st);

// multi-thread VDIF muxing (fxb_mux.cu); stream is a cudaStream_t
fxb_status vdif_mux(const uint8_t *dev_in, int64_t inbytes, int32_t nthreads, const int32_t *thread_ids,
                    int32_t inframebytes, int32_t fps, int32_t nbits, uint8_t *dev_out, int64_t outcap,
                    int64_t *outbytes, void *stream, std::string &err);

// DataStream control blocks (fxb_datastream.cpp): S is the station's delay model
fxb_status datastream_control(const Job &job, const DevStation &S, int s, fxb_ring *ring, int scan, int sec, int ns,
                              const double *delay_us, int64_t *offset, int32_t *nbytes, int32_t *datasec,
                              int32_t *datans, int32_t *validflags, size_t nflagint, std::string &err);

// integration output (fxb_vis.cpp)
fxb_status vis_calibrate(const Job &job, const fxb_vis_params *p, float *coreresult);
fxb_status vis_swin_write(const Job &job, const fxb_vis_params *p, const float *coreresult, const char *dir,
                          std::string &err);
fxb_status vis_pcal_write(const Job &job, const fxb_vis_params *p, const float *coreresult, const char *dir,
                          std::string &err);

// fxb_create with the context's device memory taken from a cudaMemPool_t
// (passed as void*; null: the device's default pool).  A server's pool keeps
// its memory mapped between jobs, so that creating and destroying contexts
// makes no allocation calls into the driver once the pool has grown.
fxb_ctx *create_ctx(const fxb_job_desc *desc, void *pool, fxb_status *status);

// Whether the context's next subint slot is free, i.e. whether a submit would
// start at once rather than wait for an earlier subint to finish (an error
// of the slot's event also reads as free, so that the submit reports it).
bool ctx_slot_free(fxb_ctx *ctx);
int calcstridelength(unsigned int arraylength);

}  // namespace fxb
