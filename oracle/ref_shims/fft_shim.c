/*
 * TEST INFRASTRUCTURE (oracle build only) -- never linked into the product.
 *
 * FFTW3-API shim (see fftw3.h) backed by an O(N log N) mixed-radix FP64 FFT.
 * Each axis of the 3D transform is a batch of 1D transforms whose "elements"
 * are contiguous vectors of the faster axes, so the y- and z-axis passes
 * stream whole rows.  The 1D algorithm is the self-sorting Stockham
 * formulation of Govindaraju et al., "High performance discrete Fourier
 * transforms on graphics processors" (SC 2008): at a stage of radix R with
 * Ns = product of the radices already done, butterfly j reads elements
 * j + r*N/R, applies twiddles exp(sign*2*pi*i*r*(j mod Ns)/(Ns*R)), does an
 * R-point DFT and writes element (j/Ns)*Ns*R + (j mod Ns) + r*Ns.
 * Radices 4, 2, 3, 5 have dedicated butterflies; any other prime factor uses
 * a direct R-point DFT, so every grid size the reference can choose works.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

#define MAXFAC 64

struct pspw_fftw_plan_s {
  int n[3];
  int sign;
  double *in;
  double *out;
};

static int factorize(int n, int *fac) {
  int nf = 0;
  while (n % 4 == 0) { fac[nf++] = 4; n /= 4; }
  while (n % 2 == 0) { fac[nf++] = 2; n /= 2; }
  while (n % 3 == 0) { fac[nf++] = 3; n /= 3; }
  while (n % 5 == 0) { fac[nf++] = 5; n /= 5; }
  for (int p = 7; n > 1; p += 2) {
    while (n % p == 0) { fac[nf++] = p; n /= p; }
  }
  return nf;
}

/* w[2t], w[2t+1] = cos, sin of sign*2*pi*t/n */
static double *roots(int n, int sign) {
  double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (int t = 0; t < n; t++) {
    double a = 2.0 * M_PI * (double)t / (double)n;
    w[2 * t] = cos(a);
    w[2 * t + 1] = sign * sin(a);
  }
  return w;
}

/* One Stockham stage over vector elements of length v (complex). */
static void stage(const double *x, double *y, int n, int R, int Ns, long v, int sign,
                  const double *w) {
  const int nb = n / R;
  const long vs = 2 * v; /* doubles per element */
  double cr[MAXFAC], ci[MAXFAC];
  double *ar = (double *)malloc(sizeof(double) * (size_t)R * 2);
  double *ai = ar + R;
  double *wr = (double *)malloc(sizeof(double) * (size_t)R * 2);
  double *wi = wr + R;
  /* roots of unity of order R for the general butterfly */
  double *gr = NULL, *gi = NULL;
  if (R > 5) {
    gr = (double *)malloc(sizeof(double) * (size_t)R * 2);
    gi = gr + R;
    for (int t = 0; t < R; t++) {
      gr[t] = w[2 * ((long)t * (n / R) % n)];
      gi[t] = w[2 * ((long)t * (n / R) % n) + 1];
    }
  }
  const double s3 = sqrt(0.75);
  const double c5a = cos(2.0 * M_PI / 5.0), s5a = sin(2.0 * M_PI / 5.0);
  const double c5b = cos(4.0 * M_PI / 5.0), s5b = sin(4.0 * M_PI / 5.0);
  (void)cr;
  (void)ci;
  for (int j = 0; j < nb; j++) {
    const int jm = j % Ns;
    /* twiddle r: exp(sign*2 pi i r jm / (Ns R)) = root index r*jm*(n/(Ns R)) */
    const long step = (long)jm * (n / (Ns * R));
    for (int r = 0; r < R; r++) {
      long t = ((long)r * step) % n;
      wr[r] = w[2 * t];
      wi[r] = w[2 * t + 1];
    }
    const long idxD = (long)(j / Ns) * Ns * R + jm;
    for (long e = 0; e < v; e++) {
      for (int r = 0; r < R; r++) {
        const double *src = x + ((long)j + (long)r * nb) * vs + 2 * e;
        double xr = src[0], xi = src[1];
        ar[r] = xr * wr[r] - xi * wi[r];
        ai[r] = xr * wi[r] + xi * wr[r];
      }
      double orr[MAXFAC], oi[MAXFAC];
      if (R == 2) {
        orr[0] = ar[0] + ar[1]; oi[0] = ai[0] + ai[1];
        orr[1] = ar[0] - ar[1]; oi[1] = ai[0] - ai[1];
      } else if (R == 4) {
        double t0r = ar[0] + ar[2], t0i = ai[0] + ai[2];
        double t1r = ar[0] - ar[2], t1i = ai[0] - ai[2];
        double t2r = ar[1] + ar[3], t2i = ai[1] + ai[3];
        double t3r = ar[1] - ar[3], t3i = ai[1] - ai[3];
        /* multiply t3 by sign*i */
        double u3r = -sign * t3i, u3i = sign * t3r;
        orr[0] = t0r + t2r; oi[0] = t0i + t2i;
        orr[2] = t0r - t2r; oi[2] = t0i - t2i;
        orr[1] = t1r + u3r; oi[1] = t1i + u3i;
        orr[3] = t1r - u3r; oi[3] = t1i - u3i;
      } else if (R == 3) {
        double sr = ar[1] + ar[2], si = ai[1] + ai[2];
        double dr = ar[1] - ar[2], di = ai[1] - ai[2];
        double mr = ar[0] - 0.5 * sr, mi = ai[0] - 0.5 * si;
        /* sign*i*sqrt(3)/2*(a1-a2) */
        double qr = -sign * s3 * di, qi = sign * s3 * dr;
        orr[0] = ar[0] + sr; oi[0] = ai[0] + si;
        orr[1] = mr + qr; oi[1] = mi + qi;
        orr[2] = mr - qr; oi[2] = mi - qi;
      } else if (R == 5) {
        double s1r = ar[1] + ar[4], s1i = ai[1] + ai[4];
        double d1r = ar[1] - ar[4], d1i = ai[1] - ai[4];
        double s2r = ar[2] + ar[3], s2i = ai[2] + ai[3];
        double d2r = ar[2] - ar[3], d2i = ai[2] - ai[3];
        double m1r = ar[0] + c5a * s1r + c5b * s2r, m1i = ai[0] + c5a * s1i + c5b * s2i;
        double m2r = ar[0] + c5b * s1r + c5a * s2r, m2i = ai[0] + c5b * s1i + c5a * s2i;
        /* sign*i*(s5a d1 + s5b d2) and sign*i*(s5b d1 - s5a d2) */
        double n1r = -sign * (s5a * d1i + s5b * d2i), n1i = sign * (s5a * d1r + s5b * d2r);
        double n2r = -sign * (s5b * d1i - s5a * d2i), n2i = sign * (s5b * d1r - s5a * d2r);
        orr[0] = ar[0] + s1r + s2r; oi[0] = ai[0] + s1i + s2i;
        orr[1] = m1r + n1r; oi[1] = m1i + n1i;
        orr[4] = m1r - n1r; oi[4] = m1i - n1i;
        orr[2] = m2r + n2r; oi[2] = m2i + n2i;
        orr[3] = m2r - n2r; oi[3] = m2i - n2i;
      } else {
        for (int k = 0; k < R; k++) {
          double sr = 0.0, si = 0.0;
          for (int r = 0; r < R; r++) {
            int t = (int)(((long)r * k) % R);
            sr += ar[r] * gr[t] - ai[r] * gi[t];
            si += ar[r] * gi[t] + ai[r] * gr[t];
          }
          orr[k] = sr;
          oi[k] = si;
        }
      }
      for (int r = 0; r < R; r++) {
        double *dst = y + (idxD + (long)r * Ns) * vs + 2 * e;
        dst[0] = orr[r];
        dst[1] = oi[r];
      }
    }
  }
  free(ar);
  free(wr);
  free(gr);
}

/* Transform `outer` consecutive blocks, each n elements of v complex values. */
static void fft_axis(double *data, long outer, int n, long v, int sign) {
  if (n == 1) return;
  int fac[MAXFAC];
  int nf = factorize(n, fac);
  double *w = roots(n, sign);
  const long blk = (long)n * v * 2;
  double *tmp = (double *)malloc(sizeof(double) * (size_t)blk);
  for (long o = 0; o < outer; o++) {
    double *a = data + o * blk;
    double *b = tmp;
    int Ns = 1;
    for (int f = 0; f < nf; f++) {
      stage(a, b, n, fac[f], Ns, v, sign, w);
      Ns *= fac[f];
      double *t = a;
      a = b;
      b = t;
    }
    if (a != data + o * blk) memcpy(data + o * blk, a, sizeof(double) * (size_t)blk);
  }
  free(tmp);
  free(w);
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags) {
  (void)flags;
  fftw_plan p = (fftw_plan)malloc(sizeof(struct pspw_fftw_plan_s));
  p->n[0] = n0;
  p->n[1] = n1;
  p->n[2] = n2;
  p->sign = sign;
  p->in = (double *)in;
  p->out = (double *)out;
  return p;
}

void fftw_execute(const fftw_plan p) {
  const long n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
  if (p->out != p->in) memcpy(p->out, p->in, sizeof(double) * 2 * (size_t)(n0 * n1 * n2));
  fft_axis(p->out, n0 * n1, (int)n2, 1, p->sign);
  fft_axis(p->out, n0, (int)n1, n2, p->sign);
  fft_axis(p->out, 1, (int)n0, n1 * n2, p->sign);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

void *fftw_malloc(size_t n) {
  void *ptr = NULL;
  if (posix_memalign(&ptr, 64, n ? n : 1) != 0) return NULL;
  return ptr;
}

void fftw_free(void *p) { free(p); }
