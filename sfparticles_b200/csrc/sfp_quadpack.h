// sfp_quadpack.h -- adaptive quadrature for the QED table generator, host and
// device.
//
// The reference builds its tables with scipy.integrate.quad
// (qed/rejection_sampling_tables.py:86-88, qed/optical_depth_tables.py:136-198),
// which runs QUADPACK (Piessens, de Doncker-Kapenga, Ueberhuber and Kahaner,
// "QUADPACK: a subroutine package for automatic integration", Springer 1983):
// QAGS on finite intervals and QAGI on [a, inf), with scipy's defaults
// epsabs = epsrel = 1.49e-8 and limit = 50.  quad's result is not the
// integral to full precision (where the absolute tolerance governs, e.g.
// integral_z^inf Ai for z > 26, it is 4e-5 off in relative terms), so tables
// that reproduce the reference's entries have to run the same algorithm.
// This file restates it:
//   * gk21 / gk15i: the 21-point Gauss-Kronrod rule on [a, b], and the
//     15-point rule on a subinterval of (0, 1] after x = bound + (1 - t) / t;
//     each returns the Kronrod estimate, the QUADPACK error estimate (scaled
//     |Kronrod - Gauss|, bounded below by 50 eps resabs), and |f| / |f - mean|
//     integrals;
//   * qelg: Wynn's epsilon algorithm on the sequence of partial results, with
//     QUADPACK's table of 50 + 2 entries and its error estimate from the last
//     three extrapolated values;
//   * qpsrt: the descending ordering of the subinterval errors (iord) kept
//     over the nrmax largest;
//   * qag_core: bisection of the subinterval with the largest error,
//     extrapolation once the small intervals dominate, roundoff detection
//     (iroff1..3), and the final choice between the extrapolated and the
//     summed result -- QAGS with the 21-point rule, QAGI with the 15-point
//     transformed rule.
// Arithmetic is float64; the integrand is a functor double(double).
#pragma once
#include <float.h>
#include <math.h>

#include "sfp_airy.h"
#include "sfp_gk_rules.h"

namespace sfp_quad {

constexpr int kLimit = 50;
constexpr double kEpmach = DBL_EPSILON;
constexpr double kUflow = DBL_MIN;
constexpr double kOflow = DBL_MAX;

SFP_HD double dmax(double a, double b) { return a > b ? a : b; }
SFP_HD double dmin(double a, double b) { return a < b ? a : b; }

// error estimate shared by both rules
SFP_HD double rule_error(double abserr, double resabs, double resasc) {
    if (resasc != 0.0 && abserr != 0.0) abserr = resasc * dmin(1.0, pow(200.0 * abserr / resasc, 1.5));
    if (resabs > kUflow / (50.0 * kEpmach)) abserr = dmax(kEpmach * 50.0 * resabs, abserr);
    return abserr;
}

// 21-point Gauss-Kronrod on [a, b]
template <class F>
SFP_HD void gk21(const F& f, double a, double b, double& result, double& abserr, double& resabs, double& resasc) {
    const double centr = 0.5 * (a + b), hlgth = 0.5 * (b - a), dhlgth = fabs(hlgth);
    double fv1[10], fv2[10];
    double resg = 0.0;
    const double fc = f(centr);
    double resk = sfp_gk::wgk21(10) * fc;
    resabs = fabs(resk);
    for (int j = 0; j < 5; ++j) {  // the Gauss nodes xgk[1], xgk[3], ..
        const int jtw = 2 * j + 1;
        const double absc = hlgth * sfp_gk::xgk21(jtw);
        const double f1 = f(centr - absc), f2 = f(centr + absc);
        fv1[jtw] = f1;
        fv2[jtw] = f2;
        const double fsum = f1 + f2;
        resg += sfp_gk::wg21(j) * fsum;
        resk += sfp_gk::wgk21(jtw) * fsum;
        resabs += sfp_gk::wgk21(jtw) * (fabs(f1) + fabs(f2));
    }
    for (int j = 0; j < 5; ++j) {  // the Kronrod nodes xgk[0], xgk[2], ..
        const int jtwm1 = 2 * j;
        const double absc = hlgth * sfp_gk::xgk21(jtwm1);
        const double f1 = f(centr - absc), f2 = f(centr + absc);
        fv1[jtwm1] = f1;
        fv2[jtwm1] = f2;
        const double fsum = f1 + f2;
        resk += sfp_gk::wgk21(jtwm1) * fsum;
        resabs += sfp_gk::wgk21(jtwm1) * (fabs(f1) + fabs(f2));
    }
    const double reskh = resk * 0.5;
    resasc = sfp_gk::wgk21(10) * fabs(fc - reskh);
    for (int j = 0; j < 10; ++j) resasc += sfp_gk::wgk21(j) * (fabs(fv1[j] - reskh) + fabs(fv2[j] - reskh));
    result = resk * hlgth;
    resabs *= dhlgth;
    resasc *= dhlgth;
    abserr = rule_error(fabs((resk - resg) * hlgth), resabs, resasc);
}

// 15-point Gauss-Kronrod on [a, b] of (0, 1] for the integral of f over
// [bound, inf): x = bound + (1 - t) / t, dx = dt / t^2
template <class F>
SFP_HD void gk15i(const F& f, double bound, double a, double b, double& result, double& abserr, double& resabs,
                  double& resasc) {
    const double centr = 0.5 * (a + b), hlgth = 0.5 * (b - a);
    double fv1[7], fv2[7];
    const double tabsc1 = bound + (1.0 - centr) / centr;
    const double fc = (f(tabsc1) / centr) / centr;
    double resg = sfp_gk::wg15(3) * fc;
    double resk = sfp_gk::wgk15(7) * fc;
    resabs = fabs(resk);
    for (int j = 0; j < 7; ++j) {
        const double absc = hlgth * sfp_gk::xgk15(j);
        const double absc1 = centr - absc, absc2 = centr + absc;
        const double t1 = bound + (1.0 - absc1) / absc1, t2 = bound + (1.0 - absc2) / absc2;
        const double f1 = (f(t1) / absc1) / absc1, f2 = (f(t2) / absc2) / absc2;
        fv1[j] = f1;
        fv2[j] = f2;
        const double fsum = f1 + f2;
        if (j & 1) resg += sfp_gk::wg15(j >> 1) * fsum;
        resk += sfp_gk::wgk15(j) * fsum;
        resabs += sfp_gk::wgk15(j) * (fabs(f1) + fabs(f2));
    }
    const double reskh = resk * 0.5;
    resasc = sfp_gk::wgk15(7) * fabs(fc - reskh);
    for (int j = 0; j < 7; ++j) resasc += sfp_gk::wgk15(j) * (fabs(fv1[j] - reskh) + fabs(fv2[j] - reskh));
    result = resk * hlgth;
    resasc *= hlgth;
    resabs *= hlgth;
    abserr = rule_error(fabs((resk - resg) * hlgth), resabs, resasc);
}

// Wynn's epsilon algorithm (QUADPACK qelg).  epstab[0..n-1] holds the
// current row (1-based in the book: epstab(1..n)); res3la the last three
// results; returns the extrapolated value and its error estimate.
SFP_HD void qelg(int& n, double* epstab, double& result, double& abserr, double* res3la, int& nres) {
    const int limexp = 50;
    ++nres;
    abserr = kOflow;
    result = epstab[n - 1];
    if (n < 3) {
        abserr = dmax(abserr, 5.0 * kEpmach * fabs(result));
        return;
    }
    epstab[n + 1] = epstab[n - 1];  // epstab(n+2) = epstab(n)
    const int newelm = (n - 1) / 2;
    epstab[n - 1] = kOflow;
    const int num = n;
    int k1 = n;
    for (int i = 1; i <= newelm; ++i) {
        const int k2 = k1 - 1, k3 = k1 - 2;
        const double res = epstab[k1 + 1];  // epstab(k1+2)
        const double e0 = epstab[k3 - 1], e1 = epstab[k2 - 1], e2 = res;
        const double e1abs = fabs(e1);
        const double delta2 = e2 - e1, err2 = fabs(delta2);
        const double tol2 = dmax(fabs(e2), e1abs) * kEpmach;
        const double delta3 = e1 - e0, err3 = fabs(delta3);
        const double tol3 = dmax(e1abs, fabs(e0)) * kEpmach;
        if (err2 <= tol2 && err3 <= tol3) {
            // e0, e1 and e2 are equal to within machine accuracy: convergence
            result = res;
            abserr = err2 + err3;
            abserr = dmax(abserr, 5.0 * kEpmach * fabs(result));
            return;
        }
        const double e3 = epstab[k1 - 1];
        epstab[k1 - 1] = e1;
        const double delta1 = e1 - e3, err1 = fabs(delta1);
        const double tol1 = dmax(e1abs, fabs(e3)) * kEpmach;
        if (err1 <= tol1 || err2 <= tol2 || err3 <= tol3) {
            n = i + i - 1;
            break;
        }
        const double ss = 1.0 / delta1 + 1.0 / delta2 - 1.0 / delta3;
        const double epsinf = fabs(ss * e1);
        if (epsinf <= 1e-4) {
            n = i + i - 1;
            break;
        }
        const double r = e1 + 1.0 / ss;
        epstab[k1 - 1] = r;
        k1 -= 2;
        const double error = err2 + fabs(r - e2) + err3;
        if (error <= abserr) {
            abserr = error;
            result = r;
        }
    }
    // shift the table
    if (n == limexp) n = 2 * (limexp / 2) - 1;
    int ib = (num % 2 == 0) ? 2 : 1;
    const int ie = newelm + 1;
    for (int i = 1; i <= ie; ++i) {
        const int ib2 = ib + 2;
        epstab[ib - 1] = epstab[ib2 - 1];
        ib = ib2;
    }
    if (num != n) {
        int indx = num - n + 1;
        for (int i = 1; i <= n; ++i) {
            epstab[i - 1] = epstab[indx - 1];
            ++indx;
        }
    }
    if (nres < 4) {
        res3la[nres - 1] = result;
        abserr = kOflow;
    } else {
        abserr = fabs(result - res3la[2]) + fabs(result - res3la[1]) + fabs(result - res3la[0]);
        res3la[0] = res3la[1];
        res3la[1] = res3la[2];
        res3la[2] = result;
    }
    abserr = dmax(abserr, 5.0 * kEpmach * fabs(result));
}

// QUADPACK qpsrt: keep iord (1-based subinterval numbers) in decreasing
// order of elist over its first nrmax.. entries
SFP_HD void qpsrt(int limit, int last, int& maxerr, double& ermax, const double* elist, int* iord, int& nrmax) {
    if (last <= 2) {
        iord[0] = 1;
        iord[1] = 2;
        maxerr = iord[nrmax - 1];
        ermax = elist[maxerr - 1];
        return;
    }
    const double errmax = elist[maxerr - 1];
    if (nrmax != 1) {
        const int ido = nrmax - 1;
        for (int i = 1; i <= ido; ++i) {
            const int isucc = iord[nrmax - 2];
            if (errmax <= elist[isucc - 1]) break;
            iord[nrmax - 1] = isucc;
            --nrmax;
        }
    }
    int jupbn = last;
    if (last > (limit / 2 + 2)) jupbn = limit + 3 - last;
    const double errmin = elist[last - 1];
    const int jbnd = jupbn - 1;
    const int ibeg = nrmax + 1;
    bool placed = false;
    int i = ibeg;
    if (ibeg <= jbnd) {
        for (i = ibeg; i <= jbnd; ++i) {
            const int isucc = iord[i - 1];
            if (errmax >= elist[isucc - 1]) {
                // insert errmax by traversing the list top-down, then errmin bottom-up
                iord[i - 2] = maxerr;
                int k = jbnd;
                bool done = false;
                for (int j = i; j <= jbnd; ++j) {
                    const int is2 = iord[k - 1];
                    if (errmin < elist[is2 - 1]) {
                        iord[k] = last;
                        done = true;
                        break;
                    }
                    iord[k] = is2;
                    --k;
                }
                if (!done) iord[i - 1] = last;
                placed = true;
                break;
            }
            iord[i - 2] = isucc;
        }
    }
    if (!placed) {
        iord[jbnd - 1] = maxerr;
        iord[jupbn - 1] = last;
    }
    maxerr = iord[nrmax - 1];
    ermax = elist[maxerr - 1];
}

// QAGS (rule 21, finite [a, b]) and QAGI (rule 15 after the transform,
// [a, inf)); returns the result (abserr and ier through references)
template <bool INF, class F>
SFP_HD double qag_core(const F& f, double a, double b, double epsabs, double epsrel, double& abserr, int& ier) {
    const int limit = kLimit;
    double alist[kLimit], blist[kLimit], rlist[kLimit], elist[kLimit];
    int iord[kLimit];
    double rlist2[52], res3la[3];
    ier = 0;
    double result = 0.0;
    abserr = 0.0;
    const double lo = INF ? 0.0 : a, hi = INF ? 1.0 : b;
    alist[0] = lo;
    blist[0] = hi;
    rlist[0] = 0.0;
    elist[0] = 0.0;
    iord[0] = 0;
    double defabs, resabs;
    if (INF) gk15i(f, a, lo, hi, result, abserr, defabs, resabs);
    else gk21(f, lo, hi, result, abserr, defabs, resabs);
    double dres = fabs(result);
    double errbnd = dmax(epsabs, epsrel * dres);
    int last = 1;
    rlist[0] = result;
    elist[0] = abserr;
    iord[0] = 1;
    if (abserr <= 100.0 * kEpmach * defabs && abserr > errbnd) ier = 2;
    if (limit == 1) ier = 1;
    if (ier != 0 || (abserr <= errbnd && abserr != resabs) || abserr == 0.0) return result;

    rlist2[0] = result;
    double errmax = abserr;
    int maxerr = 1;
    double area = result, errsum = abserr;
    abserr = kOflow;
    int nrmax = 1, nres = 0, numrl2 = 2, ktmin = 0;
    bool extrap = false, noext = false;
    int ierro = 0, iroff1 = 0, iroff2 = 0, iroff3 = 0;
    int ksgn = -1;
    if (dres >= (1.0 - 50.0 * kEpmach) * defabs) ksgn = 1;
    double small = 0.0, erlarg = 0.0, ertest = 0.0, correc = 0.0;
    bool to_sum = false;  // exit through the sum of the subinterval results
    for (last = 2; last <= limit; ++last) {
        // bisect the subinterval with the nrmax-th largest error estimate
        const double a1 = alist[maxerr - 1], b1 = 0.5 * (alist[maxerr - 1] + blist[maxerr - 1]);
        const double a2 = b1, b2 = blist[maxerr - 1];
        const double erlast = errmax;
        double area1, error1, area2, error2, defab1, defab2;
        if (INF) {
            gk15i(f, a, a1, b1, area1, error1, resabs, defab1);
            gk15i(f, a, a2, b2, area2, error2, resabs, defab2);
        } else {
            gk21(f, a1, b1, area1, error1, resabs, defab1);
            gk21(f, a2, b2, area2, error2, resabs, defab2);
        }
        const double area12 = area1 + area2, erro12 = error1 + error2;
        errsum = errsum + erro12 - errmax;
        area = area + area12 - rlist[maxerr - 1];
        if (defab1 != error1 && defab2 != error2) {
            if (fabs(rlist[maxerr - 1] - area12) <= 1e-5 * fabs(area12) && erro12 >= 0.99 * errmax) {
                if (extrap) ++iroff2;
                else ++iroff1;
            }
            if (last > 10 && erro12 > errmax) ++iroff3;
        }
        rlist[maxerr - 1] = area1;
        rlist[last - 1] = area2;
        errbnd = dmax(epsabs, epsrel * fabs(area));
        if (iroff1 + iroff2 >= 10 || iroff3 >= 20) ier = 2;
        if (iroff2 >= 5) ierro = 3;
        if (last == limit) ier = 1;
        if (dmax(fabs(a1), fabs(b2)) <= (1.0 + 100.0 * kEpmach) * (fabs(a2) + 1000.0 * kUflow)) ier = 4;
        if (error2 > error1) {
            alist[maxerr - 1] = a2;
            alist[last - 1] = a1;
            blist[last - 1] = b1;
            rlist[maxerr - 1] = area2;
            rlist[last - 1] = area1;
            elist[maxerr - 1] = error2;
            elist[last - 1] = error1;
        } else {
            alist[last - 1] = a2;
            blist[maxerr - 1] = b1;
            blist[last - 1] = b2;
            elist[maxerr - 1] = error1;
            elist[last - 1] = error2;
        }
        qpsrt(limit, last, maxerr, errmax, elist, iord, nrmax);
        if (errsum <= errbnd) {
            to_sum = true;
            break;
        }
        if (ier != 0) break;
        if (last == 2) {
            small = INF ? 0.375 : fabs(b - a) * 0.375;
            erlarg = errsum;
            ertest = errbnd;
            rlist2[1] = area;
            continue;
        }
        if (noext) continue;
        erlarg -= erlast;
        if (fabs(b1 - a1) > small) erlarg += erro12;
        if (!extrap) {
            // the smallest interval has the largest error: extrapolate from now on
            if (fabs(blist[maxerr - 1] - alist[maxerr - 1]) > small) continue;
            extrap = true;
            nrmax = 2;
        }
        bool go_on = false;  // a large interval still has an error above ertest: bisect it first
        if (ierro != 3 && erlarg > ertest) {
            const int id = nrmax;
            int jupbnd = last;
            if (last > (2 + limit / 2)) jupbnd = limit + 3 - last;
            for (int k = id; k <= jupbnd; ++k) {
                maxerr = iord[nrmax - 1];
                errmax = elist[maxerr - 1];
                if (fabs(blist[maxerr - 1] - alist[maxerr - 1]) > small) {
                    go_on = true;
                    break;
                }
                ++nrmax;
            }
        }
        if (go_on) continue;
        // extrapolate
        ++numrl2;
        rlist2[numrl2 - 1] = area;
        double reseps, abseps;
        qelg(numrl2, rlist2, reseps, abseps, res3la, nres);
        ++ktmin;
        if (ktmin > 5 && abserr < 1e-3 * errsum) ier = 5;
        if (abseps < abserr) {
            ktmin = 0;
            abserr = abseps;
            result = reseps;
            correc = erlarg;
            ertest = dmax(epsabs, epsrel * fabs(reseps));
            if (abserr <= ertest) break;
        }
        if (numrl2 == 1) noext = true;
        if (ier == 5) break;
        maxerr = iord[0];
        errmax = elist[maxerr - 1];
        nrmax = 1;
        extrap = false;
        small *= 0.5;
        erlarg = errsum;
    }
    if (last > limit) last = limit;
    if (!to_sum) {
        // set the final result and error estimate: the extrapolated result
        // unless the plain sum of the subintervals has the smaller relative
        // error (or no extrapolation happened)
        enum { kCompare, kDivergence, kSum, kDone } next = kDivergence;
        if (abserr == kOflow) {
            next = kSum;
        } else if (ier + ierro != 0) {
            if (ierro == 3) abserr += correc;
            if (ier == 0) ier = 3;
            if (result != 0.0 && area != 0.0) next = kCompare;
            else if (abserr > errsum) next = kSum;
            else if (area == 0.0) next = kDone;
        }
        if (next == kCompare) next = abserr / fabs(result) > errsum / fabs(area) ? kSum : kDivergence;
        if (next == kDivergence) {
            if (!(ksgn == -1 && dmax(fabs(result), fabs(area)) <= defabs * 0.01)) {
                if (0.01 > result / area || result / area > 100.0 || errsum > fabs(area)) ier = 6;
            }
            next = kDone;
        }
        if (next == kDone) {
            if (ier > 2) --ier;
            return result;
        }
    }
    result = 0.0;
    for (int k = 0; k < last; ++k) result += rlist[k];
    abserr = errsum;
    if (ier > 2) --ier;
    return result;
}

// scipy.integrate.quad(f, a, b) and quad(f, a, inf) with its defaults
template <class F>
SFP_HD double quad(const F& f, double a, double b) {
    double err;
    int ier;
    return qag_core<false>(f, a, b, 1.49e-8, 1.49e-8, err, ier);
}
template <class F>
SFP_HD double quad_inf(const F& f, double a) {
    double err;
    int ier;
    return qag_core<true>(f, a, 0.0, 1.49e-8, 1.49e-8, err, ier);
}

}  // namespace sfp_quad
