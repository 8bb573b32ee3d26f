/* ORACLE / TEST INFRASTRUCTURE.  Plain DFT behind the FFTW3 API (see fftw3.h). */
#include <stdlib.h>
#include <math.h>
#include "fftw3.h"

struct oracle_fftw_plan_s { int n, sign; fftw_complex *in, *out; };

fftw_complex* fftw_alloc_complex(size_t n) { return (fftw_complex*)calloc(n, sizeof(fftw_complex)); }
void fftw_free(void* p) { free(p); }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags)
{
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->n = n; p->sign = sign; p->in = in; p->out = out;
    return p;
}

void fftw_execute(const fftw_plan p)
{
    const int n = p->n;
    const long double tw = 2.0L * 3.14159265358979323846264338327950288L / n * p->sign;
    for (int k = 0; k < n; ++k) {
        long double re = 0.0L, im = 0.0L;
        for (int j = 0; j < n; ++j) {
            long idx = ((long)j * k) % n;
            long double c = cosl(tw * idx), s = sinl(tw * idx);
            long double xr = creal(p->in[j]), xi = cimag(p->in[j]);
            re += xr * c - xi * s;
            im += xr * s + xi * c;
        }
        p->out[k] = (double)re + I * (double)im;
    }
}

/* plans are leaked by cf.c (it overwrites p before destroying it); nothing to clean up globally */
void fftw_destroy_plan(fftw_plan p) { free(p); }
void fftw_cleanup(void) {}
