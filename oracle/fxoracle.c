/*
 * fxoracle -- CPU restatement of the DiFX FX hot path, in FP64.
 *
 * ORACLE / TEST INFRASTRUCTURE.  Only the tests, the smoke check and the
 * CPU-baseline leg of the bench load this file's library; the product
 * library never links or calls it.
 *
 * It restates, for the job subset described by include/fxb200.h (single
 * configuration, VDIF single-thread datastreams, real sampling, no pulsar
 * binning, one phase centre), the algorithm of:
 *   - the core-result layout   Configuration::populateResultLengths
 *                              (mpifxcorr/src/configuration.cpp:2212-2440)
 *   - the delay interpolator   Model::calculateDelayInterpolator
 *                              (mpifxcorr/src/model.cpp:229-299) and
 *                              Mode::setOffsets (mode.cpp:1525-1555)
 *   - VDIF decoding            mark5_unpack_with_offset
 *                              (libraries/mark5access/mark5access/
 *                              mark5_stream_unpacker.c:129-147), the VDIF
 *                              decoders and tables of format_vdif.c:74-149,
 *                              816-860, 1153-1216, 1879-1922, frame validation
 *                              format_vdif.c:4009-4056, blanker_mark5.c:282-313
 *   - the unpack window/weight Mk5Mode::unpack (mpifxcorr/src/mk5mode.cpp:104-177)
 *   - the station F stage      Mode::process (mpifxcorr/src/mode.cpp:649-1397)
 *   - the XMAC and weights     Core::processdata (core.cpp:877-972, 998-1045)
 *                              and the result merges (core.cpp:1774-1787,
 *                              1068-1086, 1266-1363)
 *   - phase cal                tones per recorded band (configuration.cpp:
 *                              1771-1846), the extractor choice (pcal.cpp:
 *                              139-191), the implicit-shift and shifting
 *                              extractors (pcal.cpp:927-1105, 494-705), fed
 *                              from Mode::process
 *                              (mode.cpp:773-787), copied band by band
 *                              (core.cpp:1124-1150)
 *   - zoom bands               parent and channel offset
 *                              (configuration.cpp:1734-1754), spectra and
 *                              autocorrelations as views into the parent band
 *                              (mode.cpp:169-208, 380-398), weights from the
 *                              parent band (core.cpp:1311-1322)
 *
 * Integer and index decisions (frame validity, sample offsets, nearest
 * sample, integer delay, weights, channel order) follow the reference's
 * double-precision expressions term by term.  The floating-point signal path
 * (rotators, FFT, products, sums) is evaluated in double with exact
 * sin/cos, so the result is the reference's algorithm without its FP32
 * rounding: the FP64 oracle the FP32 and tensor-core forms are checked against.
 *
 * Compile with -ffp-contract=off so that the double expressions that decide
 * integers are evaluated exactly as written.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/fxb200.h"

#define FLAGS_PER_INT 30                     /* mpifxcorr/src/mpifxcorr.h:39 */
#define HIMAG 3.3359f                        /* mark5_stream.h:75, format_vdif.c:48 */
#define TWO_PI_D 6.28318530717958647692
#define MAXBAND 256

typedef struct { double re, im; } dcx;

typedef struct {
	int npoly, order, interval;
	double poly0;
	double *coeffs;
} oracle_poly;

typedef struct fxo_job {
	int nfreq, nstation, nbaseline;
	fxb_freq *freqs;
	/* stations */
	int *nbits, *payload, *header, *nband;
	int *mux;                                         /* INTERLACEDVDIF: per-band weights */
	int *cplx;                                        /* complex (single-sideband) sampling */
	int **band_freq;
	char **band_pol;
	/* per band: clock offset and R/L delta (us), phase offset (degrees), LO
	 * offset (Hz) of the band's recorded frequency (configuration.cpp:1641-1672) */
	double **bclk, **bdclk, **bphase, **blooff;
	int *nzoom;
	int **zoom_freq, **zoom_parent, **zoom_choff;   /* parent: recorded band index */
	/* phase cal per station and recorded band: tones, bins (0: the dummy
	 * extractor's zeros), first tone bin and bin step */
	double *pcal_interval, *pcal_base;
	int **pc_ntones, **pc_nbins, **pc_first, **pc_step;
	int **pc_shift;       /* shifting extractor: the rotation's offset (Hz), else 0 */
	int64_t *pcoff;       /* core-result offset of each station's tones, or -1 */
	oracle_poly *poly;
	/* baselines: products grouped per freq in given order */
	int *ds1, *ds2, *nprod;
	int **prod_freq, **prod_b1, **prod_b2;
	int64_t subint_ns;
	int fringe_rot_order, write_autocorrs;
	/* derived */
	int blockspersend, maxproducts, bandsperautocorr;
	int *freqused, *equivused;
	int64_t corelen;
	int64_t *bloff;      /* [f*nbaseline+b] or -1 */
	int64_t *bwoff;
	int64_t *acoff, *acwoff;
	int fractionallofreq;
} fxo_job;

/* ------------------------------------------------------------ utilities */

static int ipow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void dfft(dcx *x, int n)
{
	/* in-place iterative radix-2 forward DFT, sign -1, exact twiddles */
	int i, j, k, len;
	for(i = 1, j = 0; i < n; i++)
	{
		int bit = n >> 1;
		for(; j & bit; bit >>= 1) j ^= bit;
		j ^= bit;
		if(i < j) { dcx t = x[i]; x[i] = x[j]; x[j] = t; }
	}
	for(len = 2; len <= n; len <<= 1)
	{
		int half = len >> 1;
		for(k = 0; k < half; k++)
		{
			double ang = -TWO_PI_D * (double)k / (double)len;
			double wr = cos(ang), wi = sin(ang);
			for(i = k; i < n; i += len)
			{
				dcx a = x[i], b = x[i + half];
				double tr = b.re * wr - b.im * wi, ti = b.re * wi + b.im * wr;
				x[i].re = a.re + tr; x[i].im = a.im + ti;
				x[i + half].re = a.re - tr; x[i + half].im = a.im - ti;
			}
		}
	}
}

static int station_nchan(const fxo_job *j, int s) { return j->freqs[j->band_freq[s][0]].nchan; }
/* frequency of band k of station s: recorded bands, then zoom bands
 * (Configuration::getDTotalFreqIndex) */
static int total_band_freq(const fxo_job *j, int s, int k)
{
	return k < j->nband[s] ? j->band_freq[s][k] : j->zoom_freq[s][k - j->nband[s]];
}
static double station_bw(const fxo_job *j, int s) { return j->freqs[j->band_freq[s][0]].bw_mhz; }

/* ------------------------------------------------------------ phase cal */

/* gcd of integers, and of doubles rounded to integers (mathutil.cpp:8-30) */
static long long lgcd(long a, long b)
{
	if(a == 0 || b == 0) return a > b ? a : b;
	for(;;)
	{
		a = a % b;
		if(a == 0) return b;
		b = b % a;
		if(b == 0) return a;
	}
}
static long long dgcd(double a, double b) { return lgcd((long)floor(a + 0.5), (long)floor(b + 0.5)); }

/* PCal::calcNumTones (pcal.cpp:205-222) */
static int calc_num_tones(double bw, double offset, double step)
{
	int n = 0;
	double ftone = offset;
	if(bw <= 0.0f || step <= 0.0f) return 0;
	while(ftone <= bw)
	{
		n++;
		ftone += step;
	}
	if(offset == 0.0 && ftone - step == bw)
		n--;
	return n;
}

/* Tones of one recorded band and its extractor (configuration.cpp:1776-1846,
 * lower and upper sideband, PCal::getNew pcal.cpp:139-191 with the minimum
 * frequency resolution of 1 MHz set by Mode, PCalExtractorImplicitShift
 * pcal.cpp:927-958, 1073-1086).  nbins 0: the band has no tone and reads as
 * one zero tone (the dummy extractor); nbins -1: an extractor this oracle
 * does not restate (lower sideband, trivial or shifting extractor). */
static void pcal_plan(const fxb_freq *f, double interval_d, double base_d, int *ntones, int *nbins, int *first,
                      int *step, int *shift)
{
	const float interval = (float)interval_d, base = (float)base_d;
	const double lo = f->freq_mhz, bw = f->bw_mhz;
	double tonefreq;
	int n = 0, off;
	*nbins = -1;
	*first = *step = *shift = 0;
	tonefreq = (double)((int)(lo / interval)) * interval;
	if(f->lower_sideband)
	{
		/* tones below the LO, counted downwards (configuration.cpp:1776-1811) */
		if(tonefreq == lo) tonefreq -= interval;
		if(tonefreq >= lo - bw)
			while(tonefreq - (float)(n * interval) >= lo - bw) n++;
	}
	else
	{
		if(tonefreq <= lo) tonefreq += interval;
		if(tonefreq <= lo + bw)
			while(tonefreq + (float)(n * interval) <= lo + bw) n++;
	}
	if(n == 0)
	{
		*ntones = 1;
		*nbins = 0;
		return;
	}
	*ntones = n;
	if(f->lower_sideband)
		off = (int)(long)(1e6 * lo - (1e6 * tonefreq - 0 * 1e6 * interval - 1e6 * base) + 0.5);
	else
		off = (int)(long)(1e6 * tonefreq + 0 * 1e6 * interval + 1e6 * base - 1e6 * lo + 0.5);
	{
		const double fs = 2.0 * 1e6 * bw, sp = 1e6 * interval;
		int No, Np, Nt;
		No = (int)(fs / dgcd(fs, (double)off));
		Np = (int)(fs / dgcd(fs, sp));
		Nt = calc_num_tones(1e6 * bw, (double)off, sp);
		while(fs / (2 * No) > 1e6) No *= 2;
		if(Nt == 0) { *nbins = 0; return; }
		if(off == 0 || Nt != n) return;   /* not restated */
		if((No % Np) != 0)
		{
			/* PCalExtractorShifting (pcal.cpp:494-705): rotate by the offset,
			 * fold into fs / gcd(fs, spacing) bins, tones at multiples of the
			 * step from bin 0 (every tone inside the bins) */
			int N = (int)(fs / dgcd(fs, sp));
			int st = (int)floor(N * (sp / fs));
			if((long long)(Nt - 1) * st >= N) return;
			*nbins = N;
			*step = st;
			*first = 0;
			*shift = off;
			return;
		}
		*nbins = No;
		*step = (int)floor((double)No * (sp / fs));
		*first = (int)floor((double)No * ((double)off / fs));
	}
}

/* samplegranularity (format_vdif.c:3845-3849) */
static int granularity(int nchan, int nbits)
{
	int g = 8 / (nchan * nbits);
	return g <= 0 ? 1 : g;
}

/* calcstridelength (configuration.cpp:46-58) */
static int calcstridelength(unsigned int arraylength)
{
	unsigned int guess;
	if(arraylength <= 16)
		return arraylength;
	for(guess = (unsigned int)sqrt(arraylength + 0.1); ; --guess)
		if(arraylength % guess == 0)
			return arraylength / guess;
}

/* ------------------------------------------------------------ VDIF decode */

static float lut2(int code)
{
	static const float lvl[4] = { -HIMAG, -1.0f, 1.0f, HIMAG };
	return lvl[code & 3];
}

static float lut8(int b) { return (float)((b - 128) / 3.3); }   /* format_vdif.c:122 */

/* Frame validity as mark5_stream_next_frame sees it: header word 2 nonzero
 * and invalid bit clear (format_vdif.c:4009-4056), and no fill pattern in the
 * first or last 64-bit payload word (blanker_mark5.c:282-313). */
static int frame_valid(const uint8_t *frame, int header, int payload)
{
	uint32_t w0, w2;
	uint64_t first, last;
	const uint64_t FILL = 0x1122334411223344ULL;
	memcpy(&w0, frame, 4);
	memcpy(&w2, frame + 8, 4);
	if(w2 == 0) return 0;
	if((w0 >> 31) & 1) return 0;
	memcpy(&first, frame + header, 8);
	memcpy(&last, frame + header + (payload / 8 - 1) * 8, 8);
	if(first == FILL || last == FILL) return 0;
	return 1;
}

/* mark5_unpack_with_offset for a single-thread VDIF stream: decode nsamp
 * samples per channel from sample offsetsamples.  Returns the decoder's
 * good-sample count; samples of invalid frames are 0.  For the 2- and
 * 4-channel 8-bit decoders the read position does not advance inside a
 * blanked frame (format_vdif.c:1879-1922, 1972-2020), so every sample after
 * the first blanked one in the call is blank: restated by `stuck`.
 * Reads beyond nbytes are treated as blanked (the reference reads past its
 * buffer there). */
static int vdif_unpack(const uint8_t *data, int64_t nbytes, int payload, int header, int nchan, int nbits,
                       int64_t offsetsamples, int nsamp, float *out /* [nchan][nsamp] */)
{
	int64_t framebytes = payload + header;
	int64_t framesamples = (int64_t)payload * 8 / (nchan * nbits);
	int sticky = (nbits == 8 && (nchan == 2 || nchan == 4));
	int stuck = 0, nblanksamp = 0, o, c;
	int64_t cur_frame = -1;
	int cur_valid = 0;
	for(o = 0; o < nsamp; o++)
	{
		int64_t g = offsetsamples + o;
		int64_t fr = g / framesamples;
		int64_t t = g % framesamples;
		if(fr != cur_frame)
		{
			cur_frame = fr;
			if((fr + 1) * framebytes > nbytes)
				cur_valid = 0;
			else
				cur_valid = frame_valid(data + fr * framebytes, header, payload);
		}
		if(!cur_valid)
			stuck = sticky;
		if(!cur_valid || stuck)
		{
			for(c = 0; c < nchan; c++)
				out[(int64_t)c * nsamp + o] = 0.0f;
			nblanksamp++;
			continue;
		}
		{
			const uint8_t *pl = data + fr * framebytes + header;
			for(c = 0; c < nchan; c++)
			{
				int64_t q = t * nchan + c;
				int64_t bit = q * nbits;
				int b = pl[bit >> 3];
				float v = (nbits == 2) ? lut2(b >> (bit & 7)) : lut8(b);
				out[(int64_t)c * nsamp + o] = v;
			}
		}
	}
	return nsamp - nblanksamp;
}

/* mark5_unpack_complex_with_offset for a single-thread complex VDIF stream
 * (VDIFC decoders, format_vdif.c:2369-2690 2-bit, 2829-2955 8-bit): sample t
 * of channel c is the real then the imaginary field q = 2 (t nchan + c), q + 1
 * of nbits each.  out[c][o] = (re, im).  The complex 8-bit decoders of 1, 2
 * and 4 channels do not advance inside a blanked frame: every later sample of
 * the call is blank.  mark5_unpack_complex_with_offset runs the blanker once
 * more after positioning on the first frame (mark5_stream_unpacker.c:189),
 * which only looks for fill pattern: that frame's header validity (invalid
 * bit, word 2) is not applied. */
static int vdif_unpack_complex(const uint8_t *data, int64_t nbytes, int payload, int header, int nchan, int nbits,
                               int64_t offsetsamples, int nsamp, float *out /* [nchan][nsamp][2] */)
{
	int64_t framebytes = payload + header;
	int64_t framesamples = (int64_t)payload * 8 / (nchan * nbits * 2);
	int sticky = (nbits == 8 && nchan <= 4);
	int stuck = 0, nblanksamp = 0, o, c;
	int64_t cur_frame = -1;
	int cur_valid = 0;
	for(o = 0; o < nsamp; o++)
	{
		int64_t g = offsetsamples + o;
		int64_t fr = g / framesamples;
		int64_t t = g % framesamples;
		if(fr != cur_frame)
		{
			cur_frame = fr;
			if((fr + 1) * framebytes > nbytes)
				cur_valid = 0;
			else if(o == 0)
			{
				uint64_t first, last;
				const uint64_t FILL = 0x1122334411223344ULL;
				memcpy(&first, data + fr * framebytes + header, 8);
				memcpy(&last, data + fr * framebytes + header + (payload / 8 - 1) * 8, 8);
				cur_valid = first != FILL && last != FILL;
			}
			else
				cur_valid = frame_valid(data + fr * framebytes, header, payload);
		}
		if(!cur_valid)
			stuck = sticky;
		if(!cur_valid || stuck)
		{
			for(c = 0; c < nchan; c++)
			{
				out[2 * ((int64_t)c * nsamp + o)] = 0.0f;
				out[2 * ((int64_t)c * nsamp + o) + 1] = 0.0f;
			}
			nblanksamp++;
			continue;
		}
		{
			const uint8_t *pl = data + fr * framebytes + header;
			for(c = 0; c < nchan; c++)
			{
				int64_t q = 2 * (t * nchan + c), k;
				for(k = 0; k < 2; k++)
				{
					int64_t bit = (q + k) * nbits;
					int b = pl[bit >> 3];
					out[2 * ((int64_t)c * nsamp + o) + k] = (nbits == 2) ? lut2(b >> (bit & 7)) : lut8(b);
				}
			}
		}
	}
	return nsamp - nblanksamp;
}

/* ------------------------------------------------------------ job set-up */

void fxo_destroy(fxo_job *j);

fxo_job *fxo_create(const fxb_job_desc *d)
{
	int s, b, f, p;
	fxo_job *j = (fxo_job *)calloc(1, sizeof(fxo_job));
	j->nfreq = d->nfreq;
	j->nstation = d->nstation;
	j->nbaseline = d->nbaseline;
	j->freqs = (fxb_freq *)malloc(sizeof(fxb_freq) * d->nfreq);
	memcpy(j->freqs, d->freqs, sizeof(fxb_freq) * d->nfreq);
	j->nbits = (int *)calloc(d->nstation, sizeof(int));
	j->mux = (int *)calloc(d->nstation, sizeof(int));
	j->cplx = (int *)calloc(d->nstation, sizeof(int));
	j->payload = (int *)calloc(d->nstation, sizeof(int));
	j->header = (int *)calloc(d->nstation, sizeof(int));
	j->nband = (int *)calloc(d->nstation, sizeof(int));
	j->band_freq = (int **)calloc(d->nstation, sizeof(int *));
	j->band_pol = (char **)calloc(d->nstation, sizeof(char *));
	j->poly = (oracle_poly *)calloc(d->nstation, sizeof(oracle_poly));
	j->bclk = (double **)calloc(d->nstation, sizeof(double *));
	j->bdclk = (double **)calloc(d->nstation, sizeof(double *));
	j->bphase = (double **)calloc(d->nstation, sizeof(double *));
	j->blooff = (double **)calloc(d->nstation, sizeof(double *));
	for(s = 0; s < d->nstation; s++)
	{
		const fxb_station *st = &d->stations[s];
		int k;
		j->bclk[s] = (double *)calloc(st->nband + 1, sizeof(double));
		j->bdclk[s] = (double *)calloc(st->nband + 1, sizeof(double));
		j->bphase[s] = (double *)calloc(st->nband + 1, sizeof(double));
		j->blooff[s] = (double *)calloc(st->nband + 1, sizeof(double));
		for(k = 0; k < st->nband; k++)
		{
			if(st->band_clock_us) j->bclk[s][k] = st->band_clock_us[k];
			if(st->band_clock_delta_us) j->bdclk[s][k] = st->band_clock_delta_us[k];
			if(st->band_phase_deg) j->bphase[s][k] = st->band_phase_deg[k];
			if(st->band_lo_offset_hz) j->blooff[s][k] = st->band_lo_offset_hz[k];
		}
		j->nbits[s] = st->nbits;
		j->mux[s] = st->mux_threads > 0;
		j->cplx[s] = st->complex_sampling != 0;
		j->payload[s] = st->payload_bytes;
		j->header[s] = st->header_bytes;
		j->nband[s] = st->nband;
		j->band_freq[s] = (int *)malloc(sizeof(int) * st->nband);
		j->band_pol[s] = (char *)malloc(st->nband);
		memcpy(j->band_freq[s], st->band_freq, sizeof(int) * st->nband);
		memcpy(j->band_pol[s], st->band_pol, st->nband);
	}
	/* zoom bands: the last recorded frequency (in local order) whose range
	 * holds the zoom band is its parent, the offset counts channels of the
	 * first recorded frequency (configuration.cpp:1734-1754); the parent band
	 * is the first recorded band of that frequency in the zoom band's
	 * polarisation (configuration.cpp:1245-1258) */
	j->nzoom = (int *)calloc(d->nstation, sizeof(int));
	j->zoom_freq = (int **)calloc(d->nstation, sizeof(int *));
	j->zoom_parent = (int **)calloc(d->nstation, sizeof(int *));
	j->zoom_choff = (int **)calloc(d->nstation, sizeof(int *));
	for(s = 0; s < d->nstation; s++)
	{
		const fxb_station *st = &d->stations[s];
		int z, nz = st->nzoom > 0 ? st->nzoom : 0;
		j->nzoom[s] = nz;
		j->zoom_freq[s] = (int *)calloc(nz + 1, sizeof(int));
		j->zoom_parent[s] = (int *)calloc(nz + 1, sizeof(int));
		j->zoom_choff[s] = (int *)calloc(nz + 1, sizeof(int));
		for(z = 0; z < nz; z++)
		{
			const fxb_freq *zf = &d->freqs[st->zoom_freq[z]];
			const fxb_freq *r0 = &d->freqs[st->band_freq[0]];
			double lo = zf->freq_mhz - (zf->lower_sideband ? zf->bw_mhz : 0.0), hi = lo + zf->bw_mhz;
			int k, parent = -1, off = 0;
			j->zoom_freq[s][z] = st->zoom_freq[z];
			for(k = 0; k < st->nband; k++)
			{
				int q, first = 1;
				const fxb_freq *pf = &d->freqs[st->band_freq[k]];
				double plo = pf->freq_mhz - (pf->lower_sideband ? pf->bw_mhz : 0.0), phi = plo + pf->bw_mhz;
				for(q = 0; q < k; q++) if(st->band_freq[q] == st->band_freq[k]) first = 0;
				if(!first) continue;
				if(hi <= phi && lo >= plo)
				{
					parent = st->band_freq[k];
					off = (int)(((lo - plo) / r0->bw_mhz) * r0->nchan + 0.5);
				}
			}
			j->zoom_parent[s][z] = -1;
			for(k = 0; k < st->nband && parent >= 0; k++)
				if(st->band_freq[k] == parent && st->band_pol[k] == st->zoom_pol[z])
				{
					j->zoom_parent[s][z] = k;
					break;
				}
			j->zoom_choff[s][z] = off;
		}
	}
	/* phase cal (configuration.cpp:1771-1846, pcal.cpp:139-191, 927-958) */
	j->pcal_interval = (double *)calloc((size_t)(d->nstation > 0 ? d->nstation : 1), sizeof(double));
	j->pcal_base = (double *)calloc((size_t)(d->nstation > 0 ? d->nstation : 1), sizeof(double));
	j->pc_ntones = (int **)calloc(d->nstation, sizeof(int *));
	j->pc_nbins = (int **)calloc(d->nstation, sizeof(int *));
	j->pc_first = (int **)calloc(d->nstation, sizeof(int *));
	j->pc_step = (int **)calloc(d->nstation, sizeof(int *));
	j->pc_shift = (int **)calloc(d->nstation, sizeof(int *));
	for(s = 0; s < d->nstation; s++)
	{
		const fxb_station *st = &d->stations[s];
		int k;
		j->pcal_interval[s] = st->pcal_interval_mhz;
		j->pcal_base[s] = st->pcal_base_mhz;
		j->pc_ntones[s] = (int *)calloc(st->nband, sizeof(int));
		j->pc_nbins[s] = (int *)calloc(st->nband, sizeof(int));
		j->pc_first[s] = (int *)calloc(st->nband, sizeof(int));
		j->pc_step[s] = (int *)calloc(st->nband, sizeof(int));
		j->pc_shift[s] = (int *)calloc(st->nband, sizeof(int));
		if(!(st->pcal_interval_mhz > 0))
			continue;
		for(k = 0; k < st->nband; k++)
			pcal_plan(&d->freqs[st->band_freq[k]], st->pcal_interval_mhz, st->pcal_base_mhz, &j->pc_ntones[s][k],
			          &j->pc_nbins[s][k], &j->pc_first[s][k], &j->pc_step[s][k], &j->pc_shift[s][k]);
	}
	j->ds1 = (int *)calloc(d->nbaseline, sizeof(int));
	j->ds2 = (int *)calloc(d->nbaseline, sizeof(int));
	j->nprod = (int *)calloc(d->nbaseline, sizeof(int));
	j->prod_freq = (int **)calloc(d->nbaseline, sizeof(int *));
	j->prod_b1 = (int **)calloc(d->nbaseline, sizeof(int *));
	j->prod_b2 = (int **)calloc(d->nbaseline, sizeof(int *));
	for(b = 0; b < d->nbaseline; b++)
	{
		const fxb_baseline *bl = &d->baselines[b];
		j->ds1[b] = bl->ds1;
		j->ds2[b] = bl->ds2;
		j->nprod[b] = bl->nprod;
		j->prod_freq[b] = (int *)malloc(sizeof(int) * bl->nprod);
		j->prod_b1[b] = (int *)malloc(sizeof(int) * bl->nprod);
		j->prod_b2[b] = (int *)malloc(sizeof(int) * bl->nprod);
		memcpy(j->prod_freq[b], bl->prod_freq, sizeof(int) * bl->nprod);
		memcpy(j->prod_b1[b], bl->prod_band1, sizeof(int) * bl->nprod);
		memcpy(j->prod_b2[b], bl->prod_band2, sizeof(int) * bl->nprod);
	}
	j->subint_ns = d->subint_ns;
	j->fringe_rot_order = d->fringe_rot_order;
	j->write_autocorrs = d->write_autocorrs;

	/* blockspersend (configuration.cpp:1852-1860) */
	{
		int nchan = station_nchan(j, 0);
		double bw = station_bw(j, 0);
		double fftns = 2.0 * nchan * 1000.0 / (2.0 * bw);
		j->blockspersend = (int)(d->subint_ns / fftns + 0.5);
	}

	/* getMaxProducts (configuration.cpp:843-857): max products of any baseline frequency */
	j->maxproducts = 0;
	for(b = 0; b < j->nbaseline; b++)
		for(f = 0; f < j->nfreq; f++)
		{
			int n = 0;
			for(p = 0; p < j->nprod[b]; p++)
				if(j->prod_freq[b][p] == f) n++;
			if(n > j->maxproducts) j->maxproducts = n;
		}
	j->bandsperautocorr = j->maxproducts > 2 ? 2 : 1;

	/* frequsedbybaseline and equivfrequsedbybaseline (configuration.cpp:325-368) */
	j->freqused = (int *)calloc(j->nfreq, sizeof(int));
	j->equivused = (int *)calloc(j->nfreq, sizeof(int));
	for(b = 0; b < j->nbaseline; b++)
		for(p = 0; p < j->nprod[b]; p++)
			j->freqused[j->prod_freq[b][p]] = 1;
	for(f = 0; f < j->nfreq; f++)
	{
		int k;
		if(j->freqused[f]) continue;
		for(k = 0; k < j->nfreq; k++)
		{
			double bwdiff = j->freqs[f].bw_mhz - j->freqs[k].bw_mhz;
			double freqdiff = j->freqs[f].freq_mhz - j->freqs[k].freq_mhz;
			if(j->freqs[f].lower_sideband) freqdiff -= j->freqs[f].bw_mhz;
			if(j->freqs[k].lower_sideband) freqdiff += j->freqs[k].bw_mhz;
			if(bwdiff < 1e-9 && freqdiff < 1e-9 && j->freqs[f].nchan == j->freqs[k].nchan &&
			   j->freqs[f].chans_to_avg == j->freqs[k].chans_to_avg && j->freqused[k])
				j->equivused[f] = 1;
		}
	}

	/* result layout (configuration.cpp:2300-2432), one phase centre, no bins */
	{
		int64_t idx = 0;
		j->bloff = (int64_t *)malloc(sizeof(int64_t) * j->nfreq * j->nbaseline);
		j->bwoff = (int64_t *)malloc(sizeof(int64_t) * j->nfreq * j->nbaseline);
		j->acoff = (int64_t *)malloc(sizeof(int64_t) * j->nstation);
		j->acwoff = (int64_t *)malloc(sizeof(int64_t) * j->nstation);
		for(f = 0; f < j->nfreq * j->nbaseline; f++) { j->bloff[f] = -1; j->bwoff[f] = -1; }
		for(f = 0; f < j->nfreq; f++)
		{
			if(!j->freqused[f]) continue;
			for(b = 0; b < j->nbaseline; b++)
			{
				int n = 0;
				for(p = 0; p < j->nprod[b]; p++) if(j->prod_freq[b][p] == f) n++;
				if(n == 0) continue;
				j->bloff[f * j->nbaseline + b] = idx;
				idx += (int64_t)n * j->freqs[f].nchan / j->freqs[f].chans_to_avg;
			}
		}
		for(f = 0; f < j->nfreq; f++)
		{
			if(!j->freqused[f]) continue;
			for(b = 0; b < j->nbaseline; b++)
			{
				int n = 0;
				for(p = 0; p < j->nprod[b]; p++) if(j->prod_freq[b][p] == f) n++;
				if(n == 0) continue;
				j->bwoff[f * j->nbaseline + b] = idx;
				idx += n / 2 + n % 2;
			}
		}
		for(s = 0; s < j->nstation; s++)
		{
			int k;
			j->acoff[s] = idx;
			for(k = 0; k < j->nband[s] + j->nzoom[s]; k++)
			{
				int fi = total_band_freq(j, s, k);
				if(j->freqused[fi] || j->equivused[fi])
					idx += (int64_t)j->bandsperautocorr * j->freqs[fi].nchan / j->freqs[fi].chans_to_avg;
			}
		}
		for(s = 0; s < j->nstation; s++)
		{
			int k, toadd = 0;
			j->acwoff[s] = idx;
			for(k = 0; k < j->nband[s] + j->nzoom[s]; k++)
			{
				int fi = total_band_freq(j, s, k);
				if(j->freqused[fi] || j->equivused[fi])
					toadd += j->bandsperautocorr;
			}
			toadd = (toadd + 1) / 2;
			if(toadd == 0) toadd = 1;
			idx += toadd;
		}
		/* then the phase-cal tones (configuration.cpp:2423-2431) */
		j->pcoff = (int64_t *)malloc(sizeof(int64_t) * j->nstation);
		for(s = 0; s < j->nstation; s++)
		{
			int k;
			j->pcoff[s] = -1;
			if(!(j->pcal_interval[s] > 0)) continue;
			j->pcoff[s] = idx;
			for(k = 0; k < j->nband[s]; k++)
				idx += j->pc_ntones[s][k];
		}
		j->corelen = idx;
	}

	/* fractionalLoFreq (mode.cpp:89-105), over each station's recorded freqs */
	j->fractionallofreq = 0;
	for(s = 0; s < j->nstation; s++)
	{
		int k;
		for(k = 0; k < j->nband[s]; k++)
		{
			double lo = j->freqs[j->band_freq[s][k]].freq_mhz;
			if(fabs(lo - (int)(lo + 0.5)) > 0.000000001)
				j->fractionallofreq = 1;
		}
	}
	return j;
}

void fxo_destroy(fxo_job *j)
{
	int i;
	if(!j) return;
	for(i = 0; i < j->nstation; i++)
	{
		free(j->band_freq[i]);
		free(j->band_pol[i]);
		free(j->zoom_freq[i]);
		free(j->zoom_parent[i]);
		free(j->zoom_choff[i]);
		free(j->pc_ntones[i]);
		free(j->pc_nbins[i]);
		free(j->pc_first[i]);
		free(j->pc_step[i]);
		free(j->pc_shift[i]);
		free(j->poly[i].coeffs);
	}
	for(i = 0; i < j->nbaseline; i++)
	{
		free(j->prod_freq[i]);
		free(j->prod_b1[i]);
		free(j->prod_b2[i]);
	}
	free(j->freqs); free(j->nbits); free(j->payload); free(j->header); free(j->nband); free(j->mux);
	free(j->band_freq); free(j->band_pol); free(j->poly);
	free(j->nzoom); free(j->zoom_freq); free(j->zoom_parent); free(j->zoom_choff);
	free(j->pcal_interval); free(j->pcal_base); free(j->pc_ntones); free(j->pc_nbins); free(j->pc_first);
	free(j->pc_step); free(j->pc_shift); free(j->pcoff);
	free(j->ds1); free(j->ds2); free(j->nprod); free(j->prod_freq); free(j->prod_b1); free(j->prod_b2);
	free(j->freqused); free(j->equivused); free(j->bloff); free(j->bwoff); free(j->acoff); free(j->acwoff);
	free(j);
}

int64_t fxo_core_result_length(const fxo_job *j) { return j->corelen; }
int fxo_blocks_per_send(const fxo_job *j) { return j->blockspersend; }

int fxo_layout(const fxo_job *j, int32_t *out)
{
	int k = 0, i;
	for(i = 0; i < j->nfreq * j->nbaseline; i++) out[k++] = (int32_t)j->bloff[i];
	for(i = 0; i < j->nfreq * j->nbaseline; i++) out[k++] = (int32_t)j->bwoff[i];
	for(i = 0; i < j->nstation; i++) out[k++] = (int32_t)j->acoff[i];
	for(i = 0; i < j->nstation; i++) out[k++] = (int32_t)j->acwoff[i];
	for(i = 0; i < j->nstation; i++) out[k++] = (int32_t)j->pcoff[i];
	return k;
}

int fxo_set_delay_poly(fxo_job *j, int s, int npoly, int order, double poly0_sec, int interval_s, const double *coeffs)
{
	oracle_poly *p = &j->poly[s];
	free(p->coeffs);
	p->npoly = npoly;
	p->order = order;
	p->poly0 = poly0_sec;
	p->interval = interval_s;
	p->coeffs = (double *)malloc(sizeof(double) * npoly * (order + 1));
	memcpy(p->coeffs, coeffs, sizeof(double) * npoly * (order + 1));
	return 0;
}

/* Model::calculateDelayInterpolator, order 2 (model.cpp:229-299), with the
 * timespan of Mode::setOffsets (mode.cpp:1546-1547; complex data doubles the
 * sample time and halves the span, so the real-data span serves both).
 * Returns 0 on success,
 * -1 when the time lies outside the polynomials (subint torched). */
int fxo_interpolator(const fxo_job *j, int s, int sec, int ns, double *c)
{
	const oracle_poly *p = &j->poly[s];
	double offsettime = (double)sec + ((double)ns) / 1000000000.0;
	double polyoffset = -p->poly0;
	int nchan = station_nchan(j, s);
	double sampletime = 1.0 / (2.0 * station_bw(j, s));
	double timespan = j->blockspersend * 2 * nchan * sampletime / 1e6;
	int numinc = j->blockspersend;
	int scansample, i, k;
	double ds[3], dt[3];
	if(p->npoly == 0 || !p->coeffs)
		return -1;
	scansample = (int)((offsettime + polyoffset) / (double)p->interval);
	if(scansample == p->npoly && ((offsettime + polyoffset - scansample * p->interval) < 1e-6))
		scansample--;
	if(scansample < 0 || scansample >= p->npoly)
		return -1;
	dt[1] = offsettime + polyoffset + timespan / 2.0 - scansample * p->interval;
	dt[0] = offsettime + polyoffset - scansample * p->interval;
	dt[2] = offsettime + polyoffset + timespan - scansample * p->interval;
	for(k = 0; k < 3; k++)
	{
		double tp = 1.0, sum = 0.0;
		const double *cf = p->coeffs + scansample * (p->order + 1);
		for(i = 0; i <= p->order; i++)
		{
			sum += tp * cf[i];
			tp = tp * dt[k];
		}
		ds[k] = sum;
	}
	c[0] = (2.0 * ds[0] - 4.0 * ds[1] + 2.0 * ds[2]) / (numinc * numinc);
	c[1] = (-3.0 * ds[0] + 4.0 * ds[1] - ds[2]) / numinc;
	c[2] = ds[0];
	return 0;
}

/* ------------------------------------------------------------ F stage */

typedef struct {
	int status;          /* 0 zeroed (invalid / out of range / zero weight), 1 processed */
	int nearestsample;
	float weight;
	double fracsampleerror;
	float pb[MAXBAND];   /* per-band data weights (INTERLACEDVDIF), Mk5Mode::perbandweights */
} fft_info;

/* blank_vdif_EDV4 (format_vdif.c:4699-4780) on decoded samples out[nchan][nsamp]
 * from sample offsetsamples: in every frame whose invalid bit is clear and
 * whose EDV4 validity mask lacks bit c / d (d = channels / mask length), the
 * nonzero samples of band c are zeroed and counted in invalid[c].  The
 * geometry (EDV version, mask length, channels, frame length, bits) is read
 * from the buffer's first frame, as the reference does; the C int shift
 * 1 << 31 tests mask bits 31-63, and a 32-channel "good" mask (1 << 32) - 1
 * is 0 on x86.  Frames past nbytes hold no samples (the decoder zeroed
 * them).  Headers whose geometry is not the station's blank nothing. */
static void blank_edv4(const uint8_t *data, int64_t nbytes, int payload, int header, int nchan, int nbits,
                       int64_t offsetsamples, int nsamp, float *out, int *invalid)
{
	uint32_t w2, w3, w4;
	int ml, nch, flen, spf, d, c, v = 0;
	const int64_t stride = nsamp;          /* row length of out; nsamp counts down below */
	int64_t fr, start, end, s;
	for(c = 0; c < nchan; c++) invalid[c] = 0;
	if(nbytes < 32) return;
	memcpy(&w2, data + 8, 4); memcpy(&w3, data + 12, 4); memcpy(&w4, data + 16, 4);
	ml = (int)((w4 >> 16) & 0xFF);
	if((w4 >> 24) != 4 || ml < 1 || ml > 64) return;
	nch = 1 << ((w2 >> 24) & 31);
	flen = (int)(w2 & 0xFFFFFF) * 8;
	spf = (flen - 32) * 8 / (nch * (int)(((w3 >> 26) & 31) + 1));
	d = nch / ml;
	if(d < 1 || nch != nchan || flen != payload + header || (int64_t)spf != (int64_t)payload * 8 / (nchan * nbits))
		return;
	fr = offsetsamples / spf;
	start = offsetsamples % spf;
	end = start + nsamp < spf ? start + nsamp : spf;
	for(;;)
	{
		int64_t n = end - start;
		if((fr + 1) * flen <= nbytes)
		{
			const uint8_t *h = data + fr * flen;
			uint32_t w0;
			uint64_t mask, good = nch < 32 ? (uint64_t)((1u << nch) - 1u) : 0u;
			memcpy(&w0, h, 4);
			memcpy(&mask, h + 24, 8);
			if(!((w0 >> 31) & 1) && mask != good)
				for(c = 0; c < nchan; c++)
				{
					int q = c / d;
					int keep = q < 31 ? (int)((mask >> q) & 1) : (mask & 0xFFFFFFFF80000000ULL) != 0;
					if(keep) continue;
					for(s = 0; s < n; s++)
						if(out[(int64_t)c * stride + s + v] != 0.0f)
						{
							out[(int64_t)c * stride + s + v] = 0.0f;
							invalid[c]++;
						}
				}
		}
		nsamp -= (int)n;
		if(nsamp <= 0) break;
		v += (int)n;
		fr++;
		start = 0;
		end = nsamp < spf ? nsamp : spf;
	}
}

/* Mode::process for station s, FFT index i (mode.cpp:649-1397, orders 0-2,
 * real-sampled USB/LSB).  spec receives [nband][nchan] complex.
 * *ups carries Mode's unpackstartsamples between calls (setData resets it). */
static fft_info mode_process(const fxo_job *j, int s, const uint8_t *buf, int64_t nbytes, int datasec, int datans,
                             const int32_t *validflags, int offsetsec, int offsetns, int invalid_subint,
                             const double *interp, int i, int *ups, dcx *spec, float *scratch, dcx *work)
{
	fft_info info = { 0, 0, 0.0f, 0.0 };
	int nchan = station_nchan(j, s);
	/* complex sampling (mode.cpp:51-59, 77-82, 140-143): nchan complex samples
	 * per FFT at bw per second; a sample holds two fields */
	const int cpl = j->cplx[s] ? 2 : 1;
	int fftchannels = j->cplx[s] ? nchan : 2 * nchan;
	int nb = j->nband[s];
	double bw = station_bw(j, s);
	double sampletime = j->cplx[s] ? 1.0 / bw : 1.0 / (2.0 * bw);    /* microseconds */
	int nbits = j->nbits[s];
	int gran = granularity(nb, nbits * cpl);
	int samplestounpack = fftchannels + (gran > 1 ? gran : 0);
	int unpacksamples = fftchannels;
	/* Mode's block bookkeeping for the range check (mode.cpp:124-139):
	 * samplesperblock = 1 for Mk5Mode */
	int bpbn = (nb * 1 * nbits * cpl) / 8, bpbd = 1;
	int asl = calcstridelength(nchan);
	double fftcentre, averagedelay, starttime, walltimesecs;
	int nearestsample, k, b;
	double fftstartmicrosec;

	if(bpbn == 0) { bpbn = 1; bpbd = 8 / (nb * nbits * cpl); }
	memset(spec, 0, sizeof(dcx) * nb * nchan);

	if(nbytes <= 1 || invalid_subint || (((validflags[i / FLAGS_PER_INT] >> (i % FLAGS_PER_INT)) & 0x01) == 0))
		return info;

	fftcentre = i + 0.5;
	averagedelay = interp[0] * fftcentre * fftcentre + interp[1] * fftcentre + interp[2];
	fftstartmicrosec = i * fftchannels * sampletime;
	starttime = (offsetsec - datasec) * 1000000.0 + ((double)((long long)offsetns - (long long)datans)) / 1000.0 + fftstartmicrosec - averagedelay;
	nearestsample = (int)(starttime / sampletime + 0.5);
	/* seconds since the job start: the scan starts with the job here
	 * (Model::getScanStartSec is 0 for it) */
	walltimesecs = offsetsec + offsetns / 1.0e9 + fftstartmicrosec / 1.0e6;
	info.nearestsample = nearestsample;
	if(nearestsample < -1 || (((int64_t)(nearestsample + fftchannels) / 1) * bpbn) / bpbd > nbytes)
		return info;

	{
		int do_unpack = 0, sampleoffset;
		if(nearestsample == -1) { nearestsample = 0; do_unpack = 1; }
		else if(nearestsample < *ups || nearestsample > *ups + unpacksamples - fftchannels) do_unpack = 1;
		if(!do_unpack)
			return info;                           /* dataweight stays 0: zeroed */
		sampleoffset = nearestsample;
		/* Mk5Mode::unpack (mk5mode.cpp:104-177) */
		{
			int munged, c, t, erased = 0;
			float good;
			*ups = sampleoffset - (sampleoffset % gran);
			if(j->cplx[s])
				good = (float)vdif_unpack_complex(buf, nbytes, j->payload[s], j->header[s], nb, nbits, *ups,
				                                  samplestounpack, scratch);
			else
				good = (float)vdif_unpack(buf, nbytes, j->payload[s], j->header[s], nb, nbits, *ups, samplestounpack,
				                          scratch);
			if(gran > 1)
			{
				munged = sampleoffset % gran;
				for(t = 0; t < munged; t++)
					for(c = 0; c < nb; c++)
						if(scratch[(int64_t)c * samplestounpack + t] != 0.0f) { scratch[(int64_t)c * samplestounpack + t] = 0.0f; erased++; }
				for(t = unpacksamples + munged; t < samplestounpack; t++)
					for(c = 0; c < nb; c++)
						if(scratch[(int64_t)c * samplestounpack + t] != 0.0f) { scratch[(int64_t)c * samplestounpack + t] = 0.0f; erased++; }
				good -= erased / (float)nb;
			}
			if(j->mux[s])
			{
				/* per-band weights (mk5mode.cpp:145-166) */
				int inv[MAXBAND], tot = 0;
				blank_edv4(buf, nbytes, j->payload[s], j->header[s], nb, nbits, *ups, samplestounpack, scratch, inv);
				for(c = 0; c < nb; c++)
				{
					info.pb[c] = (good - inv[c]) / (float)unpacksamples;
					tot += inv[c];
				}
				good -= (float)tot / (float)nb;
			}
			if(good < 0) good = 0;
			info.weight = good / (float)unpacksamples;
		}
	}
	info.nearestsample = nearestsample;
	if(!(info.weight > 0.0f))
		return info;
	info.status = 1;
	info.fracsampleerror = starttime - nearestsample * sampletime;

	{
		int off = nearestsample - *ups;
		double a = 0, bb = 0, cc = 0;
		int integerdelay = 0;
		int order = j->fringe_rot_order;
		double X1 = (double)asl / (double)fftchannels;
		if(order == 0)
			integerdelay = (int)averagedelay;
		else if(order == 1)
		{
			double d0 = interp[0] * i * i + interp[1] * i + interp[2];
			double d1 = interp[0] * (i + 0.5) * (i + 0.5) + interp[1] * (i + 0.5) + interp[2];
			double d2 = interp[0] * (i + 1) * (i + 1) + interp[1] * (i + 1) + interp[2];
			a = d2 - d0;
			bb = d0 + (d1 - (a * 0.5 + d0)) / 3.0;
			integerdelay = (int)bb;
			bb -= integerdelay;
		}
		else
		{
			a = interp[0];
			bb = interp[1] + i * interp[0] * 2.0;
			cc = interp[2] + i * interp[1] + i * i * interp[0];
			integerdelay = (int)cc;
			cc -= integerdelay;
		}

		/* one pass per recorded frequency; bands are matched to it */
		const int intwalltime = (int)walltimesecs;
		const double fracwalltime = walltimesecs - intwalltime;
		for(b = 0; b < nb; b++)
		{
			int fi = j->band_freq[s][b];
			int lsb = j->freqs[fi].lower_sideband;
			double lofreq = j->freqs[fi].freq_mhz;
			double fraclo = (lofreq - (int)lofreq) * (double)integerdelay;
			/* LO offset (mode.cpp:873-882, 932-951): the fringe phase loses
			 * looff x (sample time + wall-clock time) in turns, the integer
			 * seconds only through the offset's fractional part */
			const double looff = j->blooff[s][b];
			double fraclooff = 0.0, lowall = 0.0;
			/* fractional-sample error of this band: per-frequency clock offset,
			 * R/L delta split by polarisation (mode.cpp:1053-1059, 1099-1106,
			 * 1264-1268) */
			const double fseb = info.fracsampleerror - j->bclk[s][b] +
			                    (j->band_pol[s][b] == 'R' ? 0.5 : -0.5) * j->bdclk[s][b];
			const float *x = scratch + (int64_t)b * samplestounpack + off;
			int n, c;
			if(looff != 0.0)
			{
				fraclooff = fabs(looff) - (int)fabs(looff);
				if(looff < 0) fraclooff = -fraclooff;
				lowall = -looff * fracwalltime - (fabs(fraclooff) > (double)1e-9f ? fraclooff * intwalltime : 0.0);
			}
			if(j->cplx[s])
			{
				/* complex samples (mode.cpp:1182-1234): the rotator of the order in
				 * use (LO negated for the lower sideband, mode.cpp:899-903), an
				 * nchan-point complex FFT whose bins are the channels (upper
				 * sideband) or bin 0 then the conjugates of bins nchan-1 .. 1 */
				const double lo = lsb ? -lofreq : lofreq;
				const double flo = (lo - (int)lo) * (double)integerdelay;
				const float *xf = scratch + 2 * ((int64_t)b * samplestounpack + off);
				for(n = 0; n < fftchannels; n++)
				{
					int kk = n / asl, jj = n % asl;
					double xj = (double)jj / (double)fftchannels;
					double Xk = (double)(kk * asl) / (double)fftchannels;
					double ph;
					if(order == 1)
						ph = (xj * a + bb) * lo + Xk * a * lo;
					else
						ph = (xj * (bb + a * X1) + cc) * lo + kk * (xj * (2.0 * a * X1)) * lo
						     + (Xk * bb + Xk * Xk * a) * lo;
					if(j->fractionallofreq) ph += flo;
					if(looff != 0.0)
						ph += -looff * ((double)n * sampletime / 1e6) + lowall;
					ph = -TWO_PI_D * (ph - floor(ph));
					{
						const double xr = xf[2 * n], xi = xf[2 * n + 1], cr = cos(ph), ci = sin(ph);
						work[n].re = xr * cr - xi * ci;
						work[n].im = xr * ci + xi * cr;
					}
				}
				dfft(work, fftchannels);
				for(c = 0; c < nchan; c++)
				{
					dcx v;
					double fc, arg, cr, ci;
					if(!lsb)
						v = work[c];
					else if(c == 0)
						v = work[0];
					else
					{
						v.re = work[nchan - c].re;
						v.im = -work[nchan - c].im;
					}
					fc = lsb ? (double)(c - nchan) * bw / nchan : (double)c * bw / nchan;
					arg = TWO_PI_D * fc * fseb;
					cr = cos(arg);
					ci = sin(arg);
					spec[(int64_t)b * nchan + c].re = v.re * cr - v.im * ci;
					spec[(int64_t)b * nchan + c].im = v.re * ci + v.im * cr;
				}
				continue;
			}
			if(order == 0)
			{
				/* post-F: real FFT, fringe phase at the FFT centre (mode.cpp:1061-1070, 1157-1180) */
				double pr = (averagedelay - integerdelay) * lofreq;
				double prf;
				if(j->fractionallofreq) pr += integerdelay * (lofreq - (int)lofreq);
				pr -= walltimesecs * looff;
				prf = -TWO_PI_D * (pr - (int)pr);
				for(n = 0; n < fftchannels; n++) { work[n].re = x[n]; work[n].im = 0.0; }
				dfft(work, fftchannels);
				for(c = 0; c < nchan; c++)
				{
					dcx v = lsb ? (dcx){ work[nchan - c].re, -work[nchan - c].im } : work[c];
					double fc = lsb ? (double)(c - nchan) * bw / nchan : (double)c * bw / nchan;
					double arg = TWO_PI_D * fc * fseb + prf;
					double cr = cos(arg), ci = sin(arg);
					spec[(int64_t)b * nchan + c].re = v.re * cr - v.im * ci;
					spec[(int64_t)b * nchan + c].im = v.re * ci + v.im * cr;
				}
				continue;
			}
			for(n = 0; n < fftchannels; n++)
			{
				int kk = n / asl, jj = n % asl;
				double xj = (double)jj / (double)fftchannels;
				double Xk = (double)(kk * asl) / (double)fftchannels;
				double ph;
				if(order == 1)
					ph = (xj * a + bb) * lofreq + Xk * a * lofreq;
				else
					ph = (xj * (bb + a * X1) + cc) * lofreq + kk * (xj * (2.0 * a * X1)) * lofreq
					     + (Xk * bb + Xk * Xk * a) * lofreq;
				if(j->fractionallofreq) ph += fraclo;
				if(looff != 0.0)
					ph += -looff * ((double)n * sampletime / 1e6) + lowall;
				ph = -TWO_PI_D * (ph - floor(ph));
				work[n].re = x[n] * cos(ph);
				work[n].im = x[n] * sin(ph);
			}
			dfft(work, fftchannels);
			for(c = 0; c < nchan; c++)
			{
				dcx v = lsb ? work[nchan + c] : work[c];
				double fc = lsb ? (double)(c - nchan) * bw / nchan : (double)c * bw / nchan;
				double arg = TWO_PI_D * fc * fseb;
				double cr = cos(arg), ci = sin(arg);
				spec[(int64_t)b * nchan + c].re = v.re * cr - v.im * ci;
				spec[(int64_t)b * nchan + c].im = v.re * ci + v.im * cr;
			}
		}
		/* phase offset (mode.cpp:435-460, 1336-1347): of a frequency with two
		 * or more bands, the first two in band order, the one that is not R
		 * (the first if it is not R) is rotated by exp(+i pi phase / 360) */
		for(b = 0; b < nb; b++)
		{
			int fi = j->band_freq[s][b], q, b1 = -1, lcp, c;
			int first = 1;
			double ang, cr, ci;
			for(q = 0; q < b; q++) if(j->band_freq[s][q] == fi) first = 0;
			if(!first || j->bphase[s][b] == 0.0) continue;
			for(q = b + 1; q < nb; q++) if(j->band_freq[s][q] == fi) { b1 = q; break; }
			if(b1 < 0) continue;
			lcp = j->band_pol[s][b] == 'R' ? b1 : b;
			ang = TWO_PI_D * j->bphase[s][b] / 720.0;
			cr = cos(ang);
			ci = sin(ang);
			for(c = 0; c < nchan; c++)
			{
				dcx v = spec[(int64_t)lcp * nchan + c];
				spec[(int64_t)lcp * nchan + c].re = v.re * cr - v.im * ci;
				spec[(int64_t)lcp * nchan + c].im = v.re * ci + v.im * cr;
			}
		}
	}
	return info;
}

/* ------------------------------------------------------------ subint */

/* Correlate one subintegration and ADD it into coreresult (2*corelen
 * doubles).  Per-FFT weights are written to fftweights[s][t] when non-NULL. */
int fxo_process_subint(const fxo_job *j, const uint8_t *const *bufs, const int64_t *nbytes,
                       const int32_t *datasec, const int32_t *datans, const int32_t *const *validflags,
                       int sec, int ns, double *coreresult, float *fftweights)
{
	int S = j->nstation, B = j->nbaseline, T = j->blockspersend;
	int s, t, b, p, c;
	dcx **spec = (dcx **)calloc(S, sizeof(dcx *));
	double **acc_ac = (double **)calloc(S, sizeof(double *));     /* [band][2][nchan][2] */
	float **acw = (float **)calloc(S, sizeof(float *));           /* [band][2], float as Mode::weights */
	float *w = (float *)calloc((size_t)S * T, sizeof(float));
	float *pbw = NULL;                                            /* [s][t][band], INTERLACEDVDIF only */
	for(s = 0; s < S; s++)
		if(j->mux[s] && !pbw)
			pbw = (float *)calloc((size_t)S * T * MAXBAND, sizeof(float));
	int *ups = (int *)calloc(S, sizeof(int));
	int *badsub = (int *)calloc(S, sizeof(int));
	double (*interp)[3] = (double (*)[3])calloc(S, sizeof(double[3]));
	int maxn = 0, maxnb = 0;
	float *scratch;
	dcx *work;
	int32_t **allvalid = (int32_t **)calloc(S, sizeof(int32_t *));
	double ***pbins = (double ***)calloc(S, sizeof(double **));   /* phase-cal bins [s][band][N] */

	for(s = 0; s < S; s++)
	{
		int nchan = station_nchan(j, s);
		if(j->pcal_interval[s] > 0)
		{
			pbins[s] = (double **)calloc(j->nband[s], sizeof(double *));
			for(b = 0; b < j->nband[s]; b++)
				pbins[s][b] = (double *)calloc(2 * (j->pc_nbins[s][b] > 0 ? j->pc_nbins[s][b] : 1), sizeof(double));
		}
		if(2 * nchan + 8 > maxn) maxn = 2 * nchan + 8;
		if(j->nband[s] > maxnb) maxnb = j->nband[s];
		spec[s] = (dcx *)calloc((size_t)T * j->nband[s] * nchan, sizeof(dcx));
		acc_ac[s] = (double *)calloc((size_t)j->nband[s] * 2 * nchan * 2, sizeof(double));
		acw[s] = (float *)calloc((size_t)j->nband[s] * 2, sizeof(float));
		ups[s] = -999999999;
		badsub[s] = fxo_interpolator(j, s, sec, ns, interp[s]) != 0;
		if(!validflags || !validflags[s])
		{
			allvalid[s] = (int32_t *)malloc(sizeof(int32_t) * (T / FLAGS_PER_INT + 1));
			for(t = 0; t <= T / FLAGS_PER_INT; t++) allvalid[s][t] = 0x3FFFFFFF;
		}
	}
	scratch = (float *)malloc(sizeof(float) * (size_t)maxn * maxnb);
	work = (dcx *)malloc(sizeof(dcx) * maxn);

	/* F stage for every station and FFT (in FFT order, as one Core thread) */
	for(s = 0; s < S; s++)
	{
		int nchan = station_nchan(j, s), nb = j->nband[s];
		const int32_t *vf = allvalid[s] ? allvalid[s] : validflags[s];
		for(t = 0; t < T; t++)
		{
			dcx *sp = spec[s] + (size_t)t * nb * nchan;
			fft_info fi = mode_process(j, s, bufs[s], nbytes[s], datasec[s], datans[s], vf, sec, ns, badsub[s],
			                           interp[s], t, &ups[s], sp, scratch, work);
			w[(size_t)s * T + t] = fi.weight;
			if(pbw)
				memcpy(pbw + ((size_t)s * T + t) * MAXBAND, fi.pb, sizeof(fi.pb));
			if(fi.status != 1)
			{
				w[(size_t)s * T + t] = fi.status == 1 ? fi.weight : 0.0f;
				memset(sp, 0, sizeof(dcx) * nb * nchan);
				continue;
			}
			/* phase cal: the window's unpacked samples, binned by their sample
			 * number in the data second (datasamples + nearestsample + n)
			 * modulo the bin count (mode.cpp:773-787, pcal.cpp:1000-1050) */
			if(pbins[s])
			{
				int gran = granularity(nb, j->nbits[s]);
				int stu = 2 * nchan + (gran > 1 ? gran : 0);
				double sampletime = 1.0 / (2.0 * station_bw(j, s));
				long long a0 = (long long)(int)(datans[s] / (sampletime * 1e3) + 0.5) + fi.nearestsample;
				for(b = 0; b < nb; b++)
				{
					int N = j->pc_nbins[s][b], off = j->pc_shift[s][b];
					const float *x = scratch + (size_t)b * stu + (fi.nearestsample - ups[s]);
					long long fsi = (long long)(2e6 * station_bw(j, s) + 0.5);
					if(N <= 0) continue;
					for(c = 0; c < 2 * nchan; c++)
					{
						long long bin = (a0 + c) % N;
						if(off == 0)
							pbins[s][b][2 * bin] += x[c];
						else
						{
							/* the shifting extractor's rotator, exp(-2 pi i off a / fs) */
							double ang = -TWO_PI_D * (double)(((long long)off * ((a0 + c) % fsi)) % fsi) / (double)fsi;
							pbins[s][b][2 * bin] += x[c] * cos(ang);
							pbins[s][b][2 * bin + 1] += x[c] * sin(ang);
						}
					}
				}
			}
			/* autocorrelations (mode.cpp:1293-1308) and cross-pol autos (:1356-1369) */
			for(b = 0; b < nb; b++)
			{
				double *ac = acc_ac[s] + (size_t)b * 2 * nchan * 2;
				for(c = 0; c < nchan; c++)
				{
					dcx v = sp[(size_t)b * nchan + c];
					ac[2 * c] += v.re * v.re + v.im * v.im;
				}
				acw[s][2 * b] += j->mux[s] ? fi.pb[b] : fi.weight;
			}
			if(j->write_autocorrs)
			{
				int f;
				for(f = 0; f < j->nfreq; f++)
				{
					int idx[MAXBAND], cnt = 0;
					for(b = 0; b < nb; b++) if(j->band_freq[s][b] == f) idx[cnt++] = b;
					if(cnt > 1)
					{
						int q;
						for(q = 0; q < 2; q++)
						{
							int b0 = idx[q], b1 = idx[1 - q];
							double *ac = acc_ac[s] + ((size_t)b0 * 2 + 1) * nchan * 2;
							for(c = 0; c < nchan; c++)
							{
								dcx x0 = sp[(size_t)b0 * nchan + c], x1 = sp[(size_t)b1 * nchan + c];
								ac[2 * c] += x0.re * x1.re + x0.im * x1.im;
								ac[2 * c + 1] += x0.im * x1.re - x0.re * x1.im;
							}
							acw[s][2 * b0 + 1] += j->mux[s] ? fi.pb[b0] * fi.pb[b1] : fi.weight;
						}
					}
				}
			}
		}
	}

	/* XMAC (core.cpp:877-972) + baseline weights (core.cpp:998-1045) */
	for(b = 0; b < B; b++)
	{
		int s1 = j->ds1[b], s2 = j->ds2[b];
		int nb1 = j->nband[s1], nb2 = j->nband[s2];
		int pf = 0, lastf = -1;
		for(p = 0; p < j->nprod[b]; p++)
		{
			int f = j->prod_freq[b][p];
			int nchan = j->freqs[f].nchan, avg = j->freqs[f].chans_to_avg;
			int64_t base;
			float wsum = 0.0f;   /* float sequential sum, as core.cpp:1041 */
			if(f != lastf) { pf = 0; lastf = f; }
			base = j->bloff[f * B + b];
			/* a zoom band reads its parent's spectrum from its first channel */
			int k1 = j->prod_b1[b][p], k2 = j->prod_b2[b][p], o1 = 0, o2 = 0;
			int n1 = station_nchan(j, s1), n2 = station_nchan(j, s2);
			if(k1 >= nb1) { o1 = j->zoom_choff[s1][k1 - nb1]; k1 = j->zoom_parent[s1][k1 - nb1]; }
			if(k2 >= nb2) { o2 = j->zoom_choff[s2][k2 - nb2]; k2 = j->zoom_parent[s2][k2 - nb2]; }
			for(c = 0; c < nchan; c++)
			{
				double re = 0.0, im = 0.0;
				for(t = 0; t < T; t++)
				{
					dcx x1 = spec[s1][((size_t)t * nb1 + k1) * n1 + o1 + c];
					dcx x2 = spec[s2][((size_t)t * nb2 + k2) * n2 + o2 + c];
					re += x1.re * x2.re + x1.im * x2.im;
					im += x1.im * x2.re - x1.re * x2.im;
				}
				coreresult[2 * (base + (int64_t)pf * nchan / avg + c / avg)] += re / avg;
				coreresult[2 * (base + (int64_t)pf * nchan / avg + c / avg) + 1] += im / avg;
			}
			for(t = 0; t < T; t++)
				wsum += (j->mux[s1] ? pbw[((size_t)s1 * T + t) * MAXBAND + k1] : w[(size_t)s1 * T + t]) *
				        (j->mux[s2] ? pbw[((size_t)s2 * T + t) * MAXBAND + k2] : w[(size_t)s2 * T + t]);
			coreresult[2 * j->bwoff[f * B + b] + pf] += wsum;
			pf++;
		}
	}

	/* autocorrelations and weights into the result (core.cpp:1266-1363) */
	{
		int writecross = j->write_autocorrs && j->maxproducts > 2;
		for(s = 0; s < S; s++)
		{
			int nchan = station_nchan(j, s), nb = j->nband[s], pass;
			int64_t ridx = j->acoff[s];
			int64_t widx = j->acwoff[s] * 2;
			/* the station's averaging of its recorded bands (Mode::averageFrequency,
			 * mode.cpp:1399-1424, channelstoaverage of the first recorded band) */
			int savg = j->freqs[j->band_freq[s][0]].chans_to_avg;
			for(pass = 0; pass < (writecross ? 2 : 1); pass++)
				for(b = 0; b < nb + j->nzoom[s]; b++)
				{
					int fi = total_band_freq(j, s, b);
					int avg = j->freqs[fi].chans_to_avg;
					if(!(j->freqused[fi] || j->equivused[fi])) continue;
					if(b < nb)
					{
						double *ac = acc_ac[s] + ((size_t)b * 2 + pass) * nchan * 2;
						for(c = 0; c < nchan; c++)
						{
							coreresult[2 * (ridx + c / avg)] += ac[2 * c] / avg;
							coreresult[2 * (ridx + c / avg) + 1] += ac[2 * c + 1] / avg;
						}
						ridx += nchan / avg;
					}
					else
					{
						/* a zoom band's autocorrelation points into the parent's
						 * averaged one at choff / channelstoaverage and copies
						 * the zoom frequency's output channels (mode.cpp:389-397,
						 * core.cpp:1266-1290) */
						int z = b - nb, par = j->zoom_parent[s][z];
						int nout = j->freqs[fi].nchan / avg, first = j->zoom_choff[s][z] / savg, k;
						double *ac = acc_ac[s] + ((size_t)par * 2 + pass) * nchan * 2;
						for(k = 0; k < nout; k++)
						{
							int m = first + k;
							for(c = m * savg; c < (m + 1) * savg && c < nchan; c++)
							{
								coreresult[2 * (ridx + k)] += ac[2 * c] / savg;
								coreresult[2 * (ridx + k) + 1] += ac[2 * c + 1] / savg;
							}
						}
						ridx += nout;
					}
				}
			/* weights: a zoom band takes its parent band's (core.cpp:1311-1322) */
			for(pass = 0; pass < (writecross ? 2 : 1); pass++)
				for(b = 0; b < nb + j->nzoom[s]; b++)
				{
					int fi = total_band_freq(j, s, b);
					if(!(j->freqused[fi] || j->equivused[fi])) continue;
					coreresult[widx++] += acw[s][2 * (b < nb ? b : j->zoom_parent[s][b - nb])];
				}
		}
	}

	/* phase-cal tones: a forward DFT of the bins at the tone bins, band by
	 * band (pcal.cpp:1060-1086, core.cpp:1124-1150) */
	for(s = 0; s < S; s++)
	{
		int64_t ridx;
		if(!pbins[s]) continue;
		ridx = j->pcoff[s];
		for(b = 0; b < j->nband[s]; b++)
		{
			int N = j->pc_nbins[s][b], k;
			for(k = 0; k < j->pc_ntones[s][b]; k++)
			{
				double re = 0.0, im = 0.0;
				long long idx = (long long)j->pc_first[s][b] + (long long)k * j->pc_step[s][b];
				if(N > 0 && idx < N)
				{
					int m;
					for(m = 0; m < N; m++)
					{
						double ang = -TWO_PI_D * (double)((idx * m) % N) / (double)N;
						double zr = pbins[s][b][2 * m], zi = pbins[s][b][2 * m + 1];
						re += zr * cos(ang) - zi * sin(ang);
						im += zr * sin(ang) + zi * cos(ang);
					}
				}
				coreresult[2 * (ridx + k)] += re;
				coreresult[2 * (ridx + k) + 1] += im;
			}
			ridx += j->pc_ntones[s][b];
			free(pbins[s][b]);
		}
		free(pbins[s]);
	}
	free(pbins);

	if(fftweights)
		memcpy(fftweights, w, sizeof(float) * (size_t)S * T);
	for(s = 0; s < S; s++) { free(spec[s]); free(acc_ac[s]); free(acw[s]); free(allvalid[s]); }
	free(spec); free(acc_ac); free(acw); free(w); free(pbw); free(ups); free(badsub); free(interp); free(allvalid);
	free(scratch); free(work);
	return 0;
}

/* Mode::process for one FFT of one station: spectra [nband][nchan] complex
 * (double), the data weight and the nearest sample.  Returns 1 when the FFT
 * was processed, 0 when Mode zeroes it. */
int fxo_mode_fft(const fxo_job *j, int s, const uint8_t *buf, int64_t nbytes, int datasec, int datans,
                 const int32_t *validflags, int sec, int ns, int fftindex, double *spectra, float *weight, int *nearest)
{
	int nchan = station_nchan(j, s), nb = j->nband[s];
	double interp[3];
	int ups = -999999999, bad;
	float *scratch = (float *)malloc(sizeof(float) * (2 * nchan + 8) * nb);
	dcx *work = (dcx *)malloc(sizeof(dcx) * 2 * nchan);
	fft_info fi;
	int32_t allv[1024];
	if(!validflags)
	{
		int k;
		for(k = 0; k < 1024; k++) allv[k] = 0x3FFFFFFF;
		validflags = allv;
	}
	bad = fxo_interpolator(j, s, sec, ns, interp) != 0;
	fi = mode_process(j, s, buf, nbytes, datasec, datans, validflags, sec, ns, bad, interp, fftindex, &ups,
	                  (dcx *)spectra, scratch, work);
	*weight = fi.status == 1 ? fi.weight : 0.0f;
	if(nearest) *nearest = fi.nearestsample;
	if(fi.status != 1) memset(spectra, 0, sizeof(double) * 2 * nchan * nb);
	free(scratch);
	free(work);
	return fi.status;
}

/* Stand-alone decode with mark5_unpack_with_offset's contract. */
int fxo_vdif_unpack(const uint8_t *data, int64_t nbytes, int payload, int header, int nchan, int nbits,
                    int64_t offsetsamples, int nsamp, float *out)
{
	return vdif_unpack(data, nbytes, payload, header, nchan, nbits, offsetsamples, nsamp, out);
}
