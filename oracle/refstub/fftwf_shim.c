/* Project-written implementation of the FFTW3 single-precision calls made by
 * the reference's GENERIC vector layer (mpifxcorr/src/architecture.h.in:799-856
 * create plans, :985-1004 destroy them, :1017-1034 execute them).
 *
 * This is oracle test infrastructure: FFTW is neither vendored under the
 * reference nor installed here, so the compiled reference Mode gets its
 * transforms from this file.  Power-of-two lengths use a radix-4 Stockham
 * autosort transform (one radix-2 pass when log2(n) is odd) with twiddles
 * computed in double and stored in float, i.e. the same arithmetic class as
 * FFTW's single-precision codelets.  Other lengths fall back to a direct DFT
 * accumulated in double.  Unnormalised forward transform, sign -1, exactly
 * FFTW's convention. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"

typedef struct { float re, im; } shim_cf;

enum { SHIM_C2C = 1, SHIM_R2C = 2, SHIM_C2R = 3, SHIM_2D = 4 };

struct fftwf_plan_s
{
	int kind;
	int n, n1;          /* length; n1 = second dimension for 2-D plans */
	int sign;
	void *in, *out;
	shim_cf *tw;        /* per-stage twiddles, 3 per butterfly column */
	shim_cf *work0, *work1;
	int pow2;
};

void *fftwf_malloc(size_t n) { void *p = 0; if(posix_memalign(&p, 64, n ? n : 1) != 0) return 0; return p; }
void fftwf_free(void *p) { free(p); }
void *fftw_malloc(size_t n) { return fftwf_malloc(n); }
void fftw_free(void *p) { free(p); }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* Twiddle table for the Stockham passes: for a pass of current length len
 * (len = n, n/4, n/16, ... while len >= 4), entries w^p, w^2p, w^3p for
 * p < len/4 with w = exp(sign*2*pi*i/len). */
static shim_cf *make_twiddles(int n, int sign)
{
	int total = 0, len;
	shim_cf *tw, *t;
	for(len = n; len >= 4; len /= 4)
		total += 3 * (len / 4);
	tw = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * (total > 0 ? total : 1));
	t = tw;
	for(len = n; len >= 4; len /= 4)
	{
		int p;
		for(p = 0; p < len / 4; p++)
		{
			int k;
			for(k = 1; k <= 3; k++)
			{
				double ang = sign * 2.0 * M_PI * (double)(k * p) / (double)len;
				t->re = (float)cos(ang);
				t->im = (float)sin(ang);
				t++;
			}
		}
	}
	return tw;
}

static inline shim_cf cmul(shim_cf a, shim_cf b)
{
	shim_cf r;
	r.re = a.re * b.re - a.im * b.im;
	r.im = a.re * b.im + a.im * b.re;
	return r;
}

/* Radix-4 Stockham decimation-in-frequency; x is overwritten, result returned
 * in whichever of x/y holds it. */
static shim_cf *stockham(int n, int sign, const shim_cf *tw, shim_cf *x, shim_cf *y)
{
	int len = n, s = 1;
	const shim_cf *t = tw;
	while(len >= 4)
	{
		int m = len / 4, p, q;
		for(p = 0; p < m; p++)
		{
			shim_cf w1 = t[3 * p], w2 = t[3 * p + 1], w3 = t[3 * p + 2];
			for(q = 0; q < s; q++)
			{
				shim_cf a = x[q + s * (p + 0)];
				shim_cf b = x[q + s * (p + m)];
				shim_cf c = x[q + s * (p + 2 * m)];
				shim_cf d = x[q + s * (p + 3 * m)];
				shim_cf apc = { a.re + c.re, a.im + c.im };
				shim_cf amc = { a.re - c.re, a.im - c.im };
				shim_cf bpd = { b.re + d.re, b.im + d.im };
				shim_cf bmd = { b.re - d.re, b.im - d.im };
				/* jbmd = (sign*i)*(b-d) */
				shim_cf jbmd = { -sign * bmd.im, sign * bmd.re };
				shim_cf r0 = { apc.re + bpd.re, apc.im + bpd.im };
				shim_cf r1 = { amc.re + jbmd.re, amc.im + jbmd.im };
				shim_cf r2 = { apc.re - bpd.re, apc.im - bpd.im };
				shim_cf r3 = { amc.re - jbmd.re, amc.im - jbmd.im };
				y[q + s * (4 * p + 0)] = r0;
				y[q + s * (4 * p + 1)] = cmul(w1, r1);
				y[q + s * (4 * p + 2)] = cmul(w2, r2);
				y[q + s * (4 * p + 3)] = cmul(w3, r3);
			}
		}
		t += 3 * m;
		len = m;
		s *= 4;
		{ shim_cf *tmp = x; x = y; y = tmp; }
	}
	if(len == 2)
	{
		int q;
		for(q = 0; q < s; q++)
		{
			shim_cf a = x[q], b = x[q + s];
			y[q].re = a.re + b.re; y[q].im = a.im + b.im;
			y[q + s].re = a.re - b.re; y[q + s].im = a.im - b.im;
		}
		{ shim_cf *tmp = x; x = y; y = tmp; }
	}
	return x;
}

static void direct_dft(int n, int sign, const shim_cf *in, shim_cf *out)
{
	int k, j;
	for(k = 0; k < n; k++)
	{
		double sr = 0.0, si = 0.0;
		for(j = 0; j < n; j++)
		{
			double ang = sign * 2.0 * M_PI * (double)(((long long)j * k) % n) / (double)n;
			double c = cos(ang), s = sin(ang);
			sr += in[j].re * c - in[j].im * s;
			si += in[j].re * s + in[j].im * c;
		}
		out[k].re = (float)sr;
		out[k].im = (float)si;
	}
}

static void c2c(struct fftwf_plan_s *p, const shim_cf *in, shim_cf *out)
{
	if(p->pow2)
	{
		shim_cf *r;
		memcpy(p->work0, in, sizeof(shim_cf) * p->n);
		r = stockham(p->n, p->sign, p->tw, p->work0, p->work1);
		memcpy(out, r, sizeof(shim_cf) * p->n);
	}
	else
	{
		memcpy(p->work0, in, sizeof(shim_cf) * p->n);
		direct_dft(p->n, p->sign, p->work0, out);
	}
}

static struct fftwf_plan_s *new_plan(int kind, int n, int sign, void *in, void *out)
{
	struct fftwf_plan_s *p = (struct fftwf_plan_s *)calloc(1, sizeof(*p));
	p->kind = kind;
	p->n = n;
	p->sign = sign;
	p->in = in;
	p->out = out;
	p->pow2 = is_pow2(n);
	p->tw = p->pow2 ? make_twiddles(n, sign) : 0;
	p->work0 = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * n);
	p->work1 = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * n);
	return p;
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags)
{
	(void)flags;
	return new_plan(SHIM_C2C, n, sign, in, out);
}

fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags)
{
	(void)flags;
	return new_plan(SHIM_R2C, n, FFTW_FORWARD, in, out);
}

fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags)
{
	(void)flags;
	return new_plan(SHIM_C2R, n, FFTW_BACKWARD, in, out);
}

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags)
{
	struct fftwf_plan_s *p;
	(void)flags;
	p = new_plan(SHIM_2D, n1, sign, in, out);
	p->n1 = n0;
	return p;
}

void fftwf_execute(const fftwf_plan pc)
{
	struct fftwf_plan_s *p = (struct fftwf_plan_s *)pc;
	int i;
	switch(p->kind)
	{
	case SHIM_C2C:
		c2c(p, (const shim_cf *)p->in, (shim_cf *)p->out);
		break;
	case SHIM_R2C:
	{
		/* real input promoted to complex; keep bins 0..n/2 */
		shim_cf *tmp = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * p->n);
		shim_cf *res = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * p->n);
		const float *in = (const float *)p->in;
		for(i = 0; i < p->n; i++) { tmp[i].re = in[i]; tmp[i].im = 0.0f; }
		c2c(p, tmp, res);
		memcpy(p->out, res, sizeof(shim_cf) * (p->n / 2 + 1));
		fftwf_free(tmp);
		fftwf_free(res);
		break;
	}
	case SHIM_C2R:
	{
		/* Hermitian-extend the half spectrum, inverse transform, keep real part */
		shim_cf *tmp = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * p->n);
		shim_cf *res = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * p->n);
		const shim_cf *in = (const shim_cf *)p->in;
		float *out = (float *)p->out;
		for(i = 0; i <= p->n / 2; i++) tmp[i] = in[i];
		for(i = p->n / 2 + 1; i < p->n; i++) { tmp[i].re = in[p->n - i].re; tmp[i].im = -in[p->n - i].im; }
		c2c(p, tmp, res);
		for(i = 0; i < p->n; i++) out[i] = res[i].re;
		fftwf_free(tmp);
		fftwf_free(res);
		break;
	}
	case SHIM_2D:
	{
		/* row transforms then column transforms, n1 rows of length n */
		int r, c, rows = p->n1, cols = p->n;
		shim_cf *a = (shim_cf *)p->in, *o = (shim_cf *)p->out;
		shim_cf *col = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * rows);
		shim_cf *colout = (shim_cf *)fftwf_malloc(sizeof(shim_cf) * rows);
		struct fftwf_plan_s *cp = new_plan(SHIM_C2C, rows, p->sign, 0, 0);
		for(r = 0; r < rows; r++)
			c2c(p, a + (size_t)r * cols, o + (size_t)r * cols);
		for(c = 0; c < cols; c++)
		{
			for(r = 0; r < rows; r++) col[r] = o[(size_t)r * cols + c];
			c2c(cp, col, colout);
			for(r = 0; r < rows; r++) o[(size_t)r * cols + c] = colout[r];
		}
		fftwf_destroy_plan(cp);
		fftwf_free(col);
		fftwf_free(colout);
		break;
	}
	}
}

void fftwf_destroy_plan(fftwf_plan pc)
{
	struct fftwf_plan_s *p = (struct fftwf_plan_s *)pc;
	if(!p) return;
	fftwf_free(p->tw);
	fftwf_free(p->work0);
	fftwf_free(p->work1);
	free(p);
}
