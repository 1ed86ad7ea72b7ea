// ab_resp.cuh -- FP64 response generators shared by the template kernels and
// the candidate polisher: Fresnel integrals and the r / z response points.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace ab {

// ======================================================================
// FP64 Fresnel integrals: power series for x <= 1.8, Lentz continued
// fraction for erfc((1-i) sqrt(pi)/2 x) up to 5.5 (Numerical Recipes 2ed
// section 6.9), and above that the auxiliary functions' asymptotic series
// (Abramowitz & Stegun 7.3.27-28; C and S from f and g by 7.3.9-10), whose
// terms fall below 1e-18 within about a dozen steps there (3.6e-14 absolute
// against Cephes' fresnl over 5.5..40).
// ======================================================================
__device__ __forceinline__ void fresnel64(double xin, double *s, double *c)
{
    double x = fabs(xin), S, C;
    if (x < 1e-300) {
        S = 0.0;
        C = 0.0;
    } else if (x <= 1.8) {
        double t = 0.5 * M_PI * x * x, term = x, sc = 0.0, ss = 0.0;
        for (int k = 0; k < 200; k++) {
            double contrib = term / (2 * k + 1);
            switch (k & 3) {
                case 0: sc += contrib; break;
                case 1: ss += contrib; break;
                case 2: sc -= contrib; break;
                default: ss -= contrib; break;
            }
            term *= t / (k + 1);
            if (k > 4 && fabs(term) < 1e-18 * (fabs(sc) + fabs(ss))) break;
        }
        C = sc;
        S = ss;
    } else if (x >= 5.5) {
        const double px2 = M_PI * x * x, t = 1.0 / (px2 * px2);
        double f = 1.0, g = 1.0, c = 1.0, d = 1.0;
        for (int m = 1; m < 40; m++) {
            c *= -(double) ((4 * m - 3) * (4 * m - 1)) * t;
            d *= -(double) ((4 * m - 1) * (4 * m + 1)) * t;
            f += c;
            g += d;
            if (fabs(c) < 1e-18 && fabs(d) < 1e-18) break;
        }
        f /= M_PI * x;
        g /= M_PI * M_PI * x * x * x;
        double sp, cp;
        sincospi(0.5 * x * x, &sp, &cp);           // sin, cos(pi x^2 / 2)
        C = 0.5 + f * sp - g * cp;
        S = 0.5 - f * cp - g * sp;
    } else {
        const double fpmin = 1e-300;
        double px2 = M_PI * x * x;
        double br = 1.0, bi = -px2, cr = 1.0 / fpmin, ci = 0.0;
        double den = br * br + bi * bi;
        double dr = br / den, di = -bi / den, hr = dr, hi = di;
        for (int n = 1; n < 100000; n++) {
            double an = -(double) (2 * n - 1) * (double) (2 * n);
            br += 4.0;
            double tr = an * dr + br, ti = an * di + bi;
            den = tr * tr + ti * ti;
            dr = tr / den;
            di = -ti / den;
            den = cr * cr + ci * ci;
            cr = br + an * cr / den;
            ci = bi - an * ci / den;
            double delr = cr * dr - ci * di, deli = cr * di + ci * dr;
            double nhr = hr * delr - hi * deli, nhi = hr * deli + hi * delr;
            hr = nhr;
            hi = nhi;
            if (fabs(delr - 1.0) + fabs(deli) < 1e-16) break;
        }
        double sp, cp;
        sincospi(0.5 * x * x, &sp, &cp);             // e^{i pi x^2 / 2}
        double ar = x * (cp + sp), ai = x * (sp - cp);
        double fr = ar * hr - ai * hi, fi = ar * hi + ai * hr;
        double gr = 1.0 - fr, gi = -fi;
        C = 0.5 * (gr - gi);
        S = 0.5 * (gr + gi);
    }
    if (xin < 0.0) {
        C = -C;
        S = -S;
    }
    *s = S;
    *c = C;
}

// gen_r_response point c (src/responses.c:159-225), written with direct
// sin/cos of the exact argument instead of the trig recursion.
__device__ __forceinline__ double2 r_resp_point(double roffset, int numbetween, int numkern, int c)
{
    double rbypi = numkern / (double) (2 * numbetween) + roffset - (double) c / numbetween;
    double s, co;
    sincospi(rbypi, &s, &co);
    double r = M_PI * rbypi;
    double sinc = (r == 0.0) ? 1.0 : s / r;
    double2 v = make_double2(co * sinc, s * sinc);
    if (roffset < 1E-3 && c == numkern / 2) {
        double t = roffset * roffset;
        v = make_double2(1 - 6.579736267392905746 * t, roffset * (M_PI - 10.335425560099940058 * t));
    }
    return v;
}

// gen_z_response point c (src/responses.c:228-316)
__device__ __forceinline__ double2 z_resp_point(double roffset, int numbetween, double z, int numkern, int c)
{
    double absz = fabs(z);
    if (absz < 1E-4) return r_resp_point(roffset, numbetween, numkern, c);
    double startr = roffset - (0.5 * z), ip;
    double startroffset = (startr < 0) ? 1.0 + modf(startr, &ip) : modf(startr, &ip);
    int signz = (z < 0.0) ? -1 : 1;
    double zd = signz * M_SQRT2 / sqrt(absz);
    double cons = zd / 2.0;
    double pibyz = M_PI / z;
    startr += numkern / (double) (2 * numbetween);
    double r = startr + c * (-1.0 / numbetween);
    double yy = r * zd;
    double zz = yy + z * zd;
    double xx = pibyz * r * r;
    double sx, cx;
    sincos(xx, &sx, &cx);
    double fsy, fcy, fsz, fcz;
    fresnel64(yy, &fsy, &fcy);
    fresnel64(zz, &fsz, &fcz);
    double tr = signz * (fcz - fcy), ti = fsy - fsz;
    double2 v = make_double2((tr * cx - ti * sx) * cons, -(tr * sx + ti * cx) * cons);
    if (startroffset < 1E-3 && absz < 1E-3 && c == numkern / 2) {
        double z2 = z * z, x2 = startroffset * startroffset;
        v.x = 1.0 - 0.16449340668482264365 * z2;
        v.y = -0.5235987755982988731 * z;
        v.x += startroffset * 1.6449340668482264365 * z;
        v.y += startroffset * (M_PI - 0.5167712780049970029 * z2);
        v.x += x2 * (-6.579736267392905746 + 0.9277056288952613070 * z2);
        v.y += x2 * (3.1006276680299820175 * z);
    }
    return v;
}

}  // namespace ab
