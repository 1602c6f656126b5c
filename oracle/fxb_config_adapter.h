/* The mapping from the reference's parsed configuration to the fxb200 C ABI:
 * the code an integration into mpifxcorr compiles beside Core (it reads the
 * reference's Configuration, Mode and Model).  Here it is compiled into the
 * oracle's reference library (oracle/Makefile.ref) and exercised by the
 * tests through oracle/ref_harness.cpp.
 *
 *   FxbConfigDesc d;
 *   std::string err;
 *   if(!fxb_desc_from_configuration(config, configindex, FXB_XMAC_FP16, d, err)) ...
 *   fxb_ctx *ctx = fxb_create(&d.desc, &status);
 *   per subint (scan, sec, ns):
 *     fxb_interpolators_from_model(config, configindex, scan, sec, ns, interp);
 *     fxb_submit_subint_interp(ctx, bufs, nbytes, datasec, datans, validflags, sec, ns, interp);
 *   fxb_read_results(ctx, coreresult, 2 * coreresultlength);
 */
#ifndef FXB_CONFIG_ADAPTER_H
#define FXB_CONFIG_ADAPTER_H

#include <string>
#include <vector>

#include "configuration.h"
#include "fxb200.h"

/* An fxb_job_desc and the arrays it points into. */
struct FxbConfigDesc
{
	fxb_job_desc desc;
	std::vector<fxb_freq> freqs;
	std::vector<fxb_station> stations;
	std::vector<fxb_baseline> baselines;
	std::vector<std::vector<int32_t> > ints;     // band / zoom / product index arrays
	std::vector<std::vector<char> > pols;        // band and zoom polarisations
	std::vector<std::vector<double> > corr;      // per-band clock, delta, phase and LO offsets
};

/* Fills d for configuration configindex of config: the FREQ table
 * (configuration.cpp:1982-2052), each datastream's VDIF framing, recorded and
 * zoom bands, phase-cal comb and per-frequency corrections
 * (configuration.cpp:1433-1800; the corrections as getMode hands them to the
 * datastream's Mode, configuration.cpp:954-1016), the baseline products
 * (configuration.cpp:1059-1120), the subint, fringe-rotation order and
 * autocorrelation flag.  Returns false, with err set, for a configuration
 * outside the ABI (a non-VDIF datastream, complex double-sideband sampling). */
bool fxb_desc_from_configuration(Configuration *config, int configindex, int32_t xmac_kind, FxbConfigDesc &d,
                                 std::string &err);

/* Each datastream's delay interpolator for the subint at (scan, sec, ns), as
 * Mode::setOffsets obtains it (mode.cpp:1541-1554): interp[3 ds .. 3 ds + 2],
 * NaN in interp[3 ds] where the model has none.  Returns the number of
 * datastreams without one. */
int fxb_interpolators_from_model(Configuration *config, int configindex, int scan, int sec, int ns, double *interp);

/* Deletes a Mode that Configuration::getMode made.  With the FFTW build of
 * the vector library, the real-to-complex set-up that a fringe-rotation
 * order 0 Mode uses (architecture.h.in genericInitDFTR_f32) never assigns the
 * work-buffer pointer it is handed, and ~Mode frees that pointer
 * (mode.cpp:551): it is cleared first, so that ~Mode frees nothing it did
 * not allocate. */
class Mode;
void fxb_delete_mode(Mode *m);

#endif
