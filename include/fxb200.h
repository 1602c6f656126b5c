/*
 * fxb200 -- B200 (sm_100a) FX correlator hot path behind a plain C ABI.
 *
 * The library replaces, for one correlation configuration, the per-station
 * F stage of DiFX's mpifxcorr (Mode::process, mpifxcorr/src/mode.cpp:649-1397,
 * with Mk5Mode::unpack, mpifxcorr/src/mk5mode.cpp:104-177 and mark5access's
 * VDIF decoders) and the per-baseline cross-multiply-accumulate of
 * Core::processdata (mpifxcorr/src/core.cpp:877-972, weights :998-1045),
 * writing the reference's core-result layout
 * (Configuration::populateResultLengths, mpifxcorr/src/configuration.cpp:
 * 2212-2440).  All compute runs on the GPU; there is no CPU fallback.
 *
 * Conventions: every call returns an fxb_status and never aborts the
 * process.  Buffers passed in are borrowed for the duration of the call
 * unless stated otherwise.  One context belongs to one host thread at a time.
 */
#ifndef FXB200_H
#define FXB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FXB_API __attribute__((visibility("default")))
#else
#define FXB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
	FXB_OK = 0,
	FXB_ERR_ARG = 1,          /* invalid argument or job description */
	FXB_ERR_UNSUPPORTED = 2,  /* valid DiFX job outside what this build correlates */
	FXB_ERR_CUDA = 3,         /* CUDA runtime error (message via fxb_last_error) */
	FXB_ERR_NOMEM = 4,        /* device memory exhausted or over budget */
	FXB_ERR_STATE = 5,        /* call out of order (e.g. no delay model yet) */
	FXB_ERR_TIMEOUT = 6,      /* a bounded device wait expired */
	FXB_ERR_BUSY = 7,         /* serving: no slot free, try again */
	FXB_ERR_DATA = 8          /* subint data rejected (e.g. outside the delay model) */
} fxb_status;

/* Arithmetic of the cross-multiply stage. */
typedef enum {
	FXB_XMAC_FP32 = 0,        /* CUDA-core complex FP32 MAC (the plain FP32 form) */
	FXB_XMAC_BF16 = 1,        /* BF16 spectra, tensor-core MAC, FP32 accumulate */
	FXB_XMAC_FP8 = 2,         /* FP8 e4m3 spectra with per-(channel, station) scale */
	FXB_XMAC_FP16 = 3         /* FP16 spectra (fixed 2^-5 scale), tensor-core MAC, FP32 accumulate */
} fxb_xmac_kind;

/* One frequency-table entry (FREQ TABLE of the .input file,
 * configuration.cpp:1982-2052). */
typedef struct {
	double freq_mhz;          /* sky frequency of the band edge (LO), MHz */
	double bw_mhz;            /* bandwidth, MHz */
	int32_t nchan;            /* channels; the FFT length is 2*nchan */
	int32_t lower_sideband;   /* 0 = USB, 1 = LSB */
	int32_t chans_to_avg;     /* output channel averaging (>= 1) */
	int32_t reserved;
} fxb_freq;

/* One datastream: a single-thread VDIF stream whose channels are the
 * recorded bands (DATASTREAM TABLE, configuration.cpp:1433-1800).
 *
 * Zoom bands (ZOOM FREQ / ZOOM BAND entries, configuration.cpp:1719-1770)
 * are channel windows of a recorded band: zoom band z is the frequency-table
 * entry zoom_freq[z] in polarisation zoom_pol[z].  Its parent is the recorded
 * band of the same polarisation whose frequency range contains it, and its
 * first channel is the zoom band edge's offset into the parent, in parent
 * channels (configuration.cpp:1734-1754); its channel width must equal the
 * parent's.  A baseline product names zoom band z of a station as band index
 * nband + z.  Zoom frequencies must come after the station's recorded
 * frequencies in the frequency table (configuration.cpp:2598-2610). */
typedef struct {
	int32_t nbits;            /* 2 or 8 */
	int32_t payload_bytes;    /* VDIF payload bytes per frame */
	int32_t header_bytes;     /* 32 (16 = legacy) */
	int32_t nband;            /* recorded bands = VDIF channels */
	const int32_t *band_freq; /* [nband] frequency-table index of each band */
	const char *band_pol;     /* [nband] 'R'/'L'/'X'/'Y' */
	int32_t nzoom;            /* zoom bands (0: none; the pointers may be null) */
	int32_t mux_threads;      /* INTERLACEDVDIF: threads of one band each, muxed into the frames
	                           * passed (0: plain VDIF).  Data weights are then per band
	                           * (Mk5Mode::unpack, mk5mode.cpp:145-166): a band of a valid frame whose
	                           * header carries an EDV4 validity mask without the band's bit is
	                           * blanked; baselines weigh w1(band1) * w2(band2) (core.cpp:1032).
	                           * 2-bit only, no zoom bands, no phase cal. */
	const int32_t *zoom_freq; /* [nzoom] frequency-table index of each zoom band */
	const char *zoom_pol;     /* [nzoom] polarisation of each zoom band */
	/* Phase-cal extraction (PHASE CAL INT (MHZ), PHASE CAL BASE(MHZ);
	 * configuration.cpp:1600-1625, 1771-1846): comb tones every
	 * pcal_interval_mhz, shifted by pcal_base_mhz; 0 = off.  The tones of
	 * each recorded band, from its lowest in-band comb tone upwards, are
	 * extracted from the unpacked samples of every valid FFT (mode.cpp:773-787,
	 * pcal.cpp) and appended to the core result after the autocorrelation
	 * weights, band by band (core.cpp:1124-1150). */
	double pcal_interval_mhz;
	double pcal_base_mhz;
	/* Corrections per recorded frequency, given per band (bands of one
	 * frequency carry equal values; each pointer may be null for all zero):
	 * the DATASTREAM TABLE's "CLK OFFSET n (us)", read as offset[:delta[:phase]],
	 * and "FREQ OFFSET n (Hz)" (configuration.cpp:1641-1672).  As Mode::process
	 * applies them (mode.cpp:870-1145, 1296-1347, 435-460):
	 *  - the fractional-sample rotation of a band uses fse - offset + delta/2
	 *    when the band's polarisation is R, fse - offset - delta/2 otherwise;
	 *  - the fringe rotation subtracts LO offset x wall-clock time (seconds
	 *    since the job start) from the fringe phase in turns;
	 *  - where a frequency has two or more bands, the first two in band order
	 *    carry the phase offset: the one that is not R (the first, if neither
	 *    is) is rotated by exp(+i pi phase / 360).
	 * (The reference's VDIF Mode receives its FILTERBANK flag in the place of
	 * linear2circular, configuration.cpp:1009, so no linear-to-circular
	 * conversion happens on this path.) */
	const double *band_clock_us;       /* [nband] clock offset, us */
	const double *band_clock_delta_us; /* [nband] R/L clock delta, us */
	const double *band_phase_deg;      /* [nband] phase offset, degrees */
	const double *band_lo_offset_hz;   /* [nband] LO offset, Hz */
	/* INTERLACEDVDIF stations (mux_threads > 0) only.  mux_raw = 1: the buffers
	 * passed for this station are the DataStream's raw reads -- the threads'
	 * own frames (payload_bytes / mux_threads + header_bytes bytes each, one
	 * band per thread) interleaved in any order -- and the context places them
	 * and reads each band's samples from its thread's frame inside the F
	 * stage, with no muxed copy (frame slots, output headers, validity and
	 * dropped leading slots as VDIFMuxer, datamuxer.cpp:106-848);
	 * datasec/datans then give the time of the buffer's first frame.
	 * mux_raw = 0: the buffers hold the muxer's output (fxb_vdif_mux). */
	int32_t mux_raw;
	const int32_t *mux_thread_ids;   /* [mux_threads] VDIF thread id of band b's thread (null: 0, 1, ..) */
	/* DATA SAMPLING: 0 = REAL; 1 = COMPLEX (single sideband, "COMPLEX",
	 * "COMPLEX_IQ" or "COMPLEX_SSB", configuration.cpp:1545-1556): bw complex
	 * samples per second per band, each the real then the imaginary field of
	 * nbits (VDIFC decoders, format_vdif.c:2369-2410, 2868-2907); the FFT is a
	 * complex one of nchan points whose bins are the channels (upper sideband),
	 * or bin 0 then the conjugates of bins nchan - 1 .. 1 (lower sideband; the
	 * fringe rotation then uses -LO), mode.cpp:889-905, 1182-1234.  Fringe
	 * rotation order 1 or 2; 2-bit with at least 2 VDIF channels or 8-bit with
	 * at most 4; no zoom bands, phase cal or INTERLACEDVDIF. */
	int32_t complex_sampling;
} fxb_station;

/* One baseline (BASELINE TABLE, configuration.cpp:1059-1120): products are
 * listed frequency by frequency, in .input order. */
typedef struct {
	int32_t ds1, ds2;         /* datastream indices, ds1 < ds2 */
	int32_t nprod;
	const int32_t *prod_freq; /* [nprod] frequency-table index */
	const int32_t *prod_band1;/* [nprod] band index within ds1 (>= nband: zoom band) */
	const int32_t *prod_band2;/* [nprod] band index within ds2 (>= nband: zoom band) */
} fxb_baseline;

typedef struct {
	int32_t nfreq;
	const fxb_freq *freqs;
	int32_t nstation;
	const fxb_station *stations;
	int32_t nbaseline;
	const fxb_baseline *baselines;
	int64_t subint_ns;        /* SUBINT NANOSECONDS; a whole number of FFTs */
	int32_t fringe_rot_order; /* FRINGE ROTN ORDER: 0, 1 or 2 */
	int32_t write_autocorrs;  /* WRITE AUTOCORRS (also enables cross-pol autos) */
	int32_t xmac_kind;        /* fxb_xmac_kind */
	int32_t max_subints_in_flight; /* device staging depth, >= 1 */
} fxb_job_desc;

typedef struct fxb_ctx fxb_ctx;

/* Build a correlation context on the current CUDA device: validates the job,
 * computes the core-result layout and allocates device state.
 * Replaces Configuration::getMode + Mode::Mode + Core's result buffers
 * (configuration.cpp:954-1016, mode.cpp:43-462, core.cpp:33-197). */
FXB_API fxb_ctx *fxb_create(const fxb_job_desc *desc, fxb_status *status);
FXB_API void fxb_destroy(fxb_ctx *ctx);

/* Text of the last error seen by this context (or by fxb_create when ctx is
 * NULL).  Valid until the next call on the context. */
FXB_API const char *fxb_last_error(const fxb_ctx *ctx);

/* Delay model of one station, in the .im convention read by
 * Model (model.cpp:600-856): npoly consecutive polynomials, each of order
 * `order` (<= 5) in seconds since its own start, the first starting at
 * poly0_sec (seconds after the job start), each valid for interval_s seconds.
 * coeffs holds npoly*(order+1) values in microseconds.  The per-subint
 * quadratic interpolator is derived on the device in FP64 exactly as
 * Model::calculateDelayInterpolator does (model.cpp:229-299). */
FXB_API fxb_status fxb_set_delay_poly(fxb_ctx *ctx, int32_t station, int32_t npoly, int32_t order,
                              double poly0_sec, int32_t interval_s, const double *coeffs);

/* Correlate one subintegration (Mode::setData/setValidFlags/setOffsets then
 * Mode::process for every FFT, then the XMAC; mode.cpp:1525-1573, 649-1397,
 * core.cpp:705-1045) and accumulate it on the device.
 * bufs[s]/nbytes[s]: the station's VDIF frames (host memory) whose first
 * sample is at datasec[s] s + datans[s] ns after the job start;
 * validflags[s]: the valid-FFT bitfield (30 flags per int32, may be NULL for
 * all valid); (sec, ns): subint start after the job start.  Returns once the
 * inputs have been copied; the work completes asynchronously. */
FXB_API fxb_status fxb_submit_subint(fxb_ctx *ctx, const uint8_t *const *bufs, const int64_t *nbytes,
                             const int32_t *datasec, const int32_t *datans,
                             const int32_t *const *validflags, int32_t sec, int32_t ns);

/* As fxb_submit_subint, with each station's quadratic delay interpolator for
 * this subint given by the caller instead of derived on the device from the
 * polynomials of fxb_set_delay_poly (which then need not be set): interp[3 s
 * .. 3 s + 2] are the coefficients Mode::setOffsets obtains from
 * Model::calculateDelayInterpolator(scan, sec + ns / 1e9, subint seconds,
 * blockspersend, ..., 2, c) with 1e6 x the integer clock seconds taken from
 * c[2] (mode.cpp:1541-1549): delay(us) = c[0] i^2 + c[1] i + c[2] at FFT
 * index i.  NaN in interp[3 s] marks a station without a model for this time
 * (its subint is torched, mode.cpp:1551-1554).  This is the call an
 * integration into mpifxcorr makes, with the reference's own Model. */
FXB_API fxb_status fxb_submit_subint_interp(fxb_ctx *ctx, const uint8_t *const *bufs, const int64_t *nbytes,
                                    const int32_t *datasec, const int32_t *datans,
                                    const int32_t *const *validflags, int32_t sec, int32_t ns,
                                    const double *interp);

/* As fxb_submit_subint but with the station buffers already in device
 * memory (pointers from cudaMalloc); they must stay valid until the next
 * fxb_sync.  validflags stay in host memory. */
FXB_API fxb_status fxb_submit_subint_device(fxb_ctx *ctx, const uint8_t *const *dev_bufs, const int64_t *nbytes,
                                    const int32_t *datasec, const int32_t *datans,
                                    const int32_t *const *validflags, int32_t sec, int32_t ns);

/* Wait for all submitted work. */
FXB_API fxb_status fxb_sync(fxb_ctx *ctx);

/* Each staging slot's subint kernels are captured once into a CUDA graph and
 * replayed (default on); on = 0 launches them one by one. */
FXB_API fxb_status fxb_set_graphs(fxb_ctx *ctx, int32_t on);

/* Online autotuning of the kernels' scheduling: the next rounds x C subints
 * (C candidates, at most 6) run eagerly with every launch timed, each F-stage
 * kind trying FFT iterations per CTA (4, 2, 1) x grid order and each
 * tensor-core XMAC group its ring depths; then each keeps its fastest
 * candidate and the graphs are captured again.  No candidate changes the
 * arithmetic: results are identical whatever is chosen.  rounds = 0 stops
 * tuning (the choices made so far stay).  Without tuning, the F stage takes
 * as many FFT iterations per CTA as leave two CTAs per SM. */
FXB_API fxb_status fxb_autotune(fxb_ctx *ctx, int32_t rounds);
/* The current choices (and, after tuning, each candidate's fastest time) as
 * text, one line per F-stage kind and XMAC group; *needed = bytes with the
 * terminating 0. */
FXB_API fxb_status fxb_tuning_report(const fxb_ctx *ctx, char *buf, size_t len, size_t *needed);

/* Batches: contexts whose subints are submitted together, e.g. one context
 * per subband shape (bandwidth, channels, bits) of an observation whose
 * subbands are uneven.  Per subint every member copies its station buffers
 * on its own copy stream, then one CUDA graph launch runs the members'
 * kernels as parallel branches, one per member.  Fused (fxb_batch_set_fused;
 * where every member allows it: tensor-core forms without FP8, phase cal,
 * zoom bands, raw INTERLACEDVDIF reads or complex sampling, and FFTs of at
 * most 8192 points): the F stages of all members run as the persistent
 * launches over one work list that spans the members (the N = 2048
 * tensor-core FFT kinds as their own launches), and every XMAC group of
 * every member as one persistent launch on a second stream, beside the next
 * subint's F stage.  Results do not depend on the mode.  A
 * member takes no fxb_submit_subint of its own while it belongs to a batch;
 * its results are read and reset through the usual calls (ordered after the
 * batch's launches).  All members need the same max_subints_in_flight and
 * device; call the batch functions with that device current. */
typedef struct fxb_batch fxb_batch;
typedef struct {
	const uint8_t *const *bufs;       /* [nstation] host station buffers */
	const int64_t *nbytes;            /* [nstation] */
	const int32_t *datasec, *datans;  /* [nstation] start of each buffer */
	const int32_t *const *validflags; /* [nstation] or NULL */
} fxb_member_subint;
/* Destroy a batch before any of its members. */
FXB_API fxb_batch *fxb_batch_create(fxb_ctx *const *members, int32_t nmember, fxb_status *status);
/* data[nmember]: every member's buffers of the subint starting at (sec, ns). */
FXB_API fxb_status fxb_batch_submit(fxb_batch *batch, const fxb_member_subint *data, int32_t sec, int32_t ns);
/* As fxb_batch_submit with every station buffer in device memory (valid
 * until the next fxb_batch_sync), as fxb_submit_subint_device. */
FXB_API fxb_status fxb_batch_submit_device(fxb_batch *batch, const fxb_member_subint *data, int32_t sec, int32_t ns);
FXB_API fxb_status fxb_batch_sync(fxb_batch *batch);
FXB_API fxb_status fxb_batch_set_graphs(fxb_batch *batch, int32_t on);
/* on = 1: the fused launches where the members allow them (off by
 * default); *fused (may be NULL) = whether the next subints run fused.
 * fxb_read_spectra of a fused member reads the first slot's spectra. */
FXB_API fxb_status fxb_batch_set_fused(fxb_batch *batch, int32_t on, int32_t *fused);
/* fxb_autotune on every member (members still tuning run eagerly). */
FXB_API fxb_status fxb_batch_autotune(fxb_batch *batch, int32_t rounds);
FXB_API const char *fxb_batch_last_error(const fxb_batch *batch);
/* The cudaStream_t (as void*) of the batch's graph launches. */
FXB_API fxb_status fxb_batch_get_stream(const fxb_batch *batch, void **stream);
FXB_API void fxb_batch_destroy(fxb_batch *batch);

/* Number of complex values in the core-result buffer
 * (Configuration::getCoreResultLength). */
FXB_API fxb_status fxb_core_result_length(const fxb_ctx *ctx, int64_t *ncomplex);

/* Offsets into the core result: for f in freqs, b in baselines the baseline
 * offset (or -1), then the same for the baseline-weight offsets, then the
 * autocorrelation offset and the autocorrelation-weight offset of every
 * datastream (Configuration::getCoreResult*Offset).  out holds
 * 2*nfreq*nbaseline + 2*nstation ints; when it holds nstation more, the
 * phase-cal offset of every datastream (-1 without phase cal) follows. */
FXB_API fxb_status fxb_layout(const fxb_ctx *ctx, int32_t *out, size_t nint);

/* The same layout computed from a job description alone, without a GPU or a
 * context (Configuration::populateResultLengths,
 * configuration.cpp:2212-2440): validates the job, writes the offsets as
 * fxb_layout does and the core-result length in complex values. */
FXB_API fxb_status fxb_job_layout(const fxb_job_desc *desc, int32_t *out, size_t nint, int64_t *ncomplex);

/* Copy the accumulated core result (2*ncomplex floats) to host memory, in
 * the reference layout: cross-correlations, baseline weights,
 * autocorrelations, autocorrelation weights, phase-cal tones.  Synchronises. */
FXB_API fxb_status fxb_read_results(fxb_ctx *ctx, float *coreresult, size_t nfloats);

/* Zero the accumulators (Core::execute after each send, core.cpp:318-322). */
FXB_API fxb_status fxb_reset(fxb_ctx *ctx);

/* Device time in ms of the last subint's kernels (F stage, XMAC, total),
 * measured with CUDA events on the context's stream. */
FXB_API fxb_status fxb_last_timing(const fxb_ctx *ctx, float *fstage_ms, float *xmac_ms, float *total_ms);

/* Per-subint kernel timing: every subint records four CUDA events on the
 * stream that runs it (event-record nodes of the graph when graphs are on);
 * while timing is enabled their intervals are summed as slots come round
 * again.  fxb_timing_read synchronises and returns the number of subints
 * and the summed device time of the FP64 delay/parameter kernels (prep),
 * the F stage and the XMAC (with the FP8 quantisation and the weight
 * kernels), then clears the sums. */
FXB_API fxb_status fxb_timing_enable(fxb_ctx *ctx, int32_t on);
FXB_API fxb_status fxb_timing_read(fxb_ctx *ctx, int32_t *nsubint, double *prep_ms, double *fstage_ms,
                                   double *xmac_ms);

/* ---- integration output (Visibility::writedata / writedifx,
 * mpifxcorr/src/visibility.cpp:348-620, 716-900, 1060-1140).  A context's
 * accumulators hold the sum of every subint since fxb_reset -- the
 * reference's Visibility::addData (visibility.cpp:181-194) -- so an
 * integration is: reset, submit its subints, fxb_read_results, then the two
 * calls below on that buffer. */
typedef struct {
	double int_time_s;            /* INT TIME (SEC) of the configuration */
	int32_t start_mjd, start_sec; /* START MJD / START SECONDS of the job */
	int32_t scan_start_sec;       /* scan start, seconds after the job start */
	int32_t int_start_sec;        /* integration start within the scan: seconds */
	int32_t int_start_ns;         /*   and nanoseconds */
	int32_t config_index, source_index;
	const double *tsys;           /* [ndatastream] a-priori Tsys (TSYS), NULL: none */
	const int32_t *telescope;     /* [ndatastream] telescope index, NULL: the datastream index */
	const double *uvw;            /* [nbaseline * 3] u, v, w (m) at the integration centre, NULL: 0 */
	const char *const *names;     /* [ndatastream] station names (PCAL files), NULL: "DS<index>" */
} fxb_vis_params;
/* Amplitude-calibrate an integrated core result of the job in place:
 * baseline and autocorrelation weights normalised by the FFTs per
 * integration, products scaled to correlation coefficients, or with Tsys by
 * the band-averaged autocorrelations and the quantisation decorrelation
 * (weights stay raw); phase-cal tones scaled by their band's data weight.
 * Needs no GPU: the caller may be the process that writes the output rather
 * than the one correlating. */
FXB_API fxb_status fxb_vis_calibrate(const fxb_job_desc *desc, const fxb_vis_params *params, float *coreresult);
/* Append the calibrated integration to <dir>/DIFX_<mjd>_<sec>.s0000.b0000 as
 * SWIN records: every baseline product with weight > 0, then every
 * autocorrelation with weight > 0 (message via fxb_last_error(NULL)). */
FXB_API fxb_status fxb_vis_write_swin(const fxb_job_desc *desc, const fxb_vis_params *params, const float *coreresult,
                                      const char *dir);
/* Append the calibrated integration's phase-cal tones to
 * <dir>/PCAL_<mjd>_<sec>_<station> of every station extracting them, one line
 * per integration with a non-zero tone, the file starting with the
 * reference's comment header (Visibility::initialisePcalFiles and writedifx,
 * visibility.cpp:104-135, 928-990). */
FXB_API fxb_status fxb_vis_write_pcal(const fxb_job_desc *desc, const fxb_vis_params *params, const float *coreresult,
                                      const char *dir);

/* ---- INTERLACEDVDIF: multi-thread VDIF to the single-thread, multi-channel
 * frames the correlator takes (VDIFMuxer::deinterlace, multiplex and the
 * corner turn, mpifxcorr/src/datamuxer.cpp:106-848), on the device.  One
 * call is one read: dev_in holds inbytes of inframebytes-byte frames of the
 * threads thread_ids[nthreads] (any order; other threads are skipped), the
 * first frame giving the read's start; dev_out receives inbytes / inframebytes
 * / nthreads output frames of (inframebytes - 32) * nthreads + 32 bytes at
 * most (*outbytes: written), frames missing a thread marked invalid.
 * Synchronises the stream (a cudaStream_t, may be NULL). */
FXB_API fxb_status fxb_vdif_mux(const uint8_t *dev_in, int64_t inbytes, int32_t nthreads, const int32_t *thread_ids,
                                int32_t inframebytes, int32_t frames_per_second, int32_t nbits, uint8_t *dev_out,
                                int64_t outcap, int64_t *outbytes, void *stream);

/* ---- DataStream control blocks: which bytes of a datastream's receive ring
 * hold a subint, their time, and which of its FFTs have data
 * (DataStream::calculateControlParams, datastream.cpp:376-636, with the VDIF
 * frame alignment of VDIFDataStream::calculateControlParams,
 * vdiffile.cpp:358-485).  A ring is nseg segments of readbytes bytes (whole
 * frames), filled in time order by the caller's reader; memory past the
 * ring's end repeats its start for at least one subint, so that a subint's
 * bytes are contiguous as the reference's overflow area makes them. */
#define FXB_INVALID_SUBINT (-99999999)   /* Mode::INVALID_SUBINT (mode.h:232) */

/* One read segment (DataStream::readinfo, datastream.h:95-120). */
typedef struct {
	int32_t scan;             /* scan of the segment's data */
	int32_t sec, ns;          /* time of the segment's first frame (scanseconds, scanns) */
	int32_t readto;           /* 1 once the reader has filled (or tried to fill) the segment */
	int64_t validbytes;       /* bytes read into the segment; readbytes when full */
} fxb_segment;

typedef struct {
	int32_t nseg;             /* segments in the ring (NUM DATA SEGMENTS) */
	int32_t readbytes;        /* bytes of one segment, a whole number of frames */
	int32_t atsegment;        /* in/out: the segment the previous subint started in (0 at the start) */
	int32_t keepreading;      /* 1 while the reader may still fill segments */
	int32_t lastvalid;        /* with keepreading 0: the last segment the reader filled */
	int32_t guard_ns;         /* GUARD NANOSECONDS of the configuration (when the .input leaves it 0
	                           * the reference derives it from the delay model's largest rate,
	                           * configuration.cpp:2741-2795: pass that value) */
	const fxb_segment *seg;   /* [nseg] */
} fxb_ring;

/* The control block of subint (scan, sec, ns) for station `station` of the
 * context's job: *offset = the byte of the ring where the subint's frames
 * start, *nbytes = how many bytes to hand to fxb_submit_subint,
 * *datasec / *datans = the time of that byte, validflags[nflagint] = the
 * valid-FFT bits (30 per int, FLAGS_PER_INT); *datasec = FXB_INVALID_SUBINT
 * when the ring holds no data for the subint (it is then submitted with
 * nbytes 0 or skipped).  delay_us = the station's delays (us, integer clock
 * seconds removed) at the subint's start and end, or NULL to evaluate the
 * context's delay model as Model::calculateDelayInterpolator does at order 0
 * (model.cpp:229-269).  FXB_ERR_STATE: while keepreading, no segment reaches
 * the subint yet (the reference's main thread waits for its reader there);
 * read further and ask again.  Host arithmetic only: no device work. */
FXB_API fxb_status fxb_datastream_control(fxb_ctx *ctx, int32_t station, fxb_ring *ring, int32_t scan, int32_t sec,
                                          int32_t ns, const double *delay_us, int64_t *offset, int32_t *nbytes,
                                          int32_t *datasec, int32_t *datans, int32_t *validflags, size_t nflagint);

/* The same from a job description and the station's delay model (the
 * arguments of fxb_set_delay_poly), without a GPU or a context. */
FXB_API fxb_status fxb_job_datastream_control(const fxb_job_desc *desc, int32_t station, int32_t npoly, int32_t order,
                                              double poly0_sec, int32_t interval_s, const double *coeffs,
                                              fxb_ring *ring, int32_t scan, int32_t sec, int32_t ns,
                                              const double *delay_us, int64_t *offset, int32_t *nbytes,
                                              int32_t *datasec, int32_t *datans, int32_t *validflags,
                                              size_t nflagint);

/* Page-locked host memory for station buffers: fxb_submit_subint copies from
 * it asynchronously at full link speed, where a pageable buffer is staged by
 * the driver on the calling thread.  Free with fxb_host_free. */
FXB_API void *fxb_host_alloc(size_t bytes, fxb_status *status);
FXB_API void fxb_host_free(void *p);

/* The cudaStream_t (as void*) on which the context launches its kernels,
 * so that callers can order their own work and events against it. */
FXB_API fxb_status fxb_get_stream(const fxb_ctx *ctx, void **stream);

/* As fxb_read_results, but the core result is written asynchronously (on
 * the context's stream) into device memory, e.g. for a cross-GPU reduction
 * of time-sharded subints. */
FXB_API fxb_status fxb_read_results_device(fxb_ctx *ctx, float *dev_out, size_t nfloats);

/* F-stage output of the last subint for one frequency: spectra[t][row][c]
 * complex (FP32, converted from the XMAC operand type), rows = the
 * (station, band) inputs recording that frequency in station order.
 * Debug/parity access; synchronises. */
FXB_API fxb_status fxb_read_spectra(fxb_ctx *ctx, int32_t freq, float *out, size_t nfloats,
                            int32_t *nfft, int32_t *nrow);

/* Per-FFT station weights of the last subint: weights[s][t] (the data
 * weight of Mode::getDataWeight).  Synchronises. */
FXB_API fxb_status fxb_read_fft_weights(fxb_ctx *ctx, float *out, size_t nfloats);

/* Decode VDIF payload samples on the GPU, the call Mk5Mode::unpack makes
 * into mark5access (mark5_unpack_with_offset,
 * libraries/mark5access/mark5access/mark5_stream_unpacker.c:129-147, with the
 * decoders of format_vdif.c and the blanker of blanker_mark5.c:282-313).
 * data: nbytes of back-to-back VDIF frames (host memory); out: [nchan][nsamp]
 * floats (host memory); *good: good-sample count as mark5access returns it. */
FXB_API fxb_status fxb_vdif_unpack(const uint8_t *data, int64_t nbytes, int32_t payload_bytes, int32_t header_bytes,
                           int32_t nchan, int32_t nbits, int64_t offsetsamples, int32_t nsamp,
                           float *out, int32_t *good);

/* Per-station F stage that allocates nothing (no counterpart in the
 * reference: DiFX's Mode allocates its buffers in its constructor).  For
 * callers that cannot call cudaMalloc -- a process whose device memory is all
 * pre-assigned to its own pool, or a real-time pipeline that forbids
 * allocation after set-up.  The caller owns every buffer: dev_vdif (the
 * station's VDIF frames, device memory), dev_spectra (output,
 * [fft][band][nchan] complex FP32, device memory) and dev_weights (output,
 * per-FFT data weight, device memory, may be NULL).  All intermediates live
 * in one fixed file-scope device array of under 1 MiB, so the call refuses
 * (FXB_ERR_UNSUPPORTED) jobs beyond 8192 FFTs per subint, 131072 frames per
 * buffer or 4096 channels.  The array is shared by every call on a device:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * Its device address is looked up on the first call on each device, which
 * should therefore come before any stream capture.  Arguments otherwise mean
 * what they mean for fxb_job_desc, fxb_set_delay_poly and fxb_submit_subint
 * (one station).  The subint holds T = subint_ns / (2 nchan x 1000 / (2 bw_mhz))
 * FFTs (returned in *nfft when nfft is not NULL): spectra_floats must be at
 * least T x nband x nchan x 2 and, with dev_weights, weight_floats at least
 * T, else FXB_ERR_ARG.  INTERLACEDVDIF stations (mux_threads != 0) and
 * stations with nonzero per-band clock, phase or LO offsets are refused with
 * FXB_ERR_UNSUPPORTED; zoom bands and phase-cal tones of the
 * station are not produced.  Returns when the work on `stream` has
 * completed. */
FXB_API fxb_status fxb_station_fstage_noalloc(const fxb_freq *freqs, int32_t nfreq, const fxb_station *station,
                                              int32_t fringe_rot_order, int64_t subint_ns, int32_t npoly,
                                              int32_t order, double poly0_sec, int32_t interval_s,
                                              const double *coeffs, const uint8_t *dev_vdif, int64_t nbytes,
                                              int32_t datasec, int32_t datans, const int32_t *validflags,
                                              int32_t sec, int32_t ns, float *dev_spectra, size_t spectra_floats,
                                              float *dev_weights, size_t weight_floats, int32_t *nfft,
                                              void *stream);

/* ------------------------------------------------------------------ serving
 * A request loop that takes correlation jobs of different shapes as they
 * arrive (the boundary's fxb_server_* calls; no counterpart in mpifxcorr,
 * whose FxManager schedules one configuration at a time, fxmanager.cpp:
 * 334-337).  Each admitted job gets its own context (device state and
 * accumulators resident until it completes) and stream; the server's worker
 * thread submits the subints of every admitted job in turn, so the work of
 * jobs that arrive while others run overlaps on the device.  Jobs are
 * admitted in arrival order while their device footprint fits the HBM budget
 * and fewer than max_active run. */
typedef struct fxb_server fxb_server;

typedef struct {
	const fxb_job_desc *desc;
	/* delay model of each station, as for fxb_set_delay_poly */
	const int32_t *poly_npoly;       /* [nstation] */
	const int32_t *poly_order;       /* [nstation] */
	const double *poly0_sec;         /* [nstation] */
	const int32_t *poly_interval;    /* [nstation] */
	const double *const *poly_coeffs;/* [nstation] */
	int32_t nsubint;
	const uint8_t *const *bufs;      /* [nsubint * nstation] host VDIF of each subint and station */
	const int64_t *nbytes;           /* [nsubint * nstation] */
	const int32_t *datasec, *datans; /* [nsubint * nstation] first-sample times */
	const int32_t *subsec, *subns;   /* [nsubint] subint start times */
	float *coreresult;               /* out: 2 * corelen floats, written when the job completes */
} fxb_job_request;

/* Device footprint of a job (bytes) as used by admission. */
FXB_API fxb_status fxb_job_footprint(const fxb_job_desc *desc, size_t *bytes);

/* Start a server on `device` with an HBM budget (bytes) for the admitted
 * jobs and at most max_active jobs on the device at once. */
FXB_API fxb_server *fxb_server_create(int32_t device, size_t hbm_budget_bytes, int32_t max_active,
                                      fxb_status *status);
/* Queue a job.  Every array of the request (and the job description) is
 * borrowed until the job has completed; returns its id. */
FXB_API fxb_status fxb_server_submit(fxb_server *srv, const fxb_job_request *req, uint64_t *job_id);
/* state: 0 queued, 1 running, 2 done, 3 failed; latency_ms = submit to
 * completion (done jobs). */
FXB_API fxb_status fxb_server_poll(fxb_server *srv, uint64_t job_id, int32_t *state, double *latency_ms);
/* Block until the job is done or failed, or timeout_s passes
 * (FXB_ERR_TIMEOUT). */
FXB_API fxb_status fxb_server_wait(fxb_server *srv, uint64_t job_id, double timeout_s);
/* Where a done job's latency went, phase_ms[5]: queued (submit to admission),
 * context creation, subint submission (start to last subint queued), drain
 * (last subint queued to completion seen), result read and release. */
FXB_API fxb_status fxb_server_job_times(fxb_server *srv, uint64_t job_id, double *phase_ms);
/* Completed jobs, p50 / p99 latency (ms), data seconds correlated, and wall
 * seconds from the first submit to the last completion. */
FXB_API fxb_status fxb_server_stats(fxb_server *srv, int32_t *ncompleted, double *p50_ms, double *p99_ms,
                                    double *data_seconds, double *wall_seconds);
/* Text of the server's last error (e.g. of a failed job). */
FXB_API const char *fxb_server_last_error(const fxb_server *srv);
/* Finish the running jobs, fail the queued ones, stop the worker. */
FXB_API void fxb_server_destroy(fxb_server *srv);

#ifdef __cplusplus
}
#endif

#endif /* FXB200_H */
