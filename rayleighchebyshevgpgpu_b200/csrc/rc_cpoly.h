// rc_cpoly.h -- design of the Lanczos "C" filter polynomial (host scalars).
//
// Same quantities as LanczosCpoly (LanczosCpoly.h:112-708), computed independently:
//   P_m(x) = U_m(1 - 2x)/(m+1), i.e. with sin^2(theta/2) = x, P_m = sin((m+1)theta)/((m+1) sin theta);
//   evaluated by the three-term recurrence b_k = (2-4x) b_{k-1} - b_{k-2} (LanczosCpoly.h:234-270).
//   XStar(m)      = the x in (0, x_1) with P_m(x) = |min of P_m between its first two roots|
//                   (getXStar, :285-293); x_1 is the first root.
//   UpperXStar(m) = the next-to-largest root (1 + cos(2 pi/(m+1)))/2 (getUpperXStar/getPmNextToLastRoot,
//                   :295-305, :363-369); degrees 0, 1, 2 use the reference's fixed defaults.
//   starDegree/starBound: the smallest degree m (< polyDegreeMax) with
//                   XStar/UpperXStar * (lambdaBound + shift) < lambdaStar + shift, and the stretched
//                   bound mapping lambdaStar onto XStar (getStarDegreeAndSpectralRadius, :498-555).
// The roots of P_m' and of P_m(x) = y are found here by bisection (the reference uses secant
// iterations to 1e-12); both converge to the same points well below that tolerance.
#pragma once
#include <cmath>
#include <vector>

namespace rcb {

class CPoly {
public:
    static double pm(long m, double x) {
        if (m <= 0) return 1.0;
        const double c = 2.0 - 4.0 * x;
        double bkm2 = 1.0, bkm1 = c;
        for (long k = 2; k <= m; ++k) {
            const double bk = c * bkm1 - bkm2;
            bkm2 = bkm1;
            bkm1 = bk;
        }
        return bkm1 / (double)(m + 1);
    }

    // x of the first interior extremum of P_m (m >= 2): zero of dP/dtheta between the first two
    // roots theta = pi/(m+1) and 2 pi/(m+1), where
    //   dP/dtheta ~ (m+1) cos((m+1) theta) sin(theta) - sin((m+1) theta) cos(theta).
    static double first_extremum(long m) {
        const double pi = 3.14159265358979323846;
        const double mp = (double)(m + 1);
        auto f = [&](double t) { return mp * std::cos(mp * t) * std::sin(t) - std::sin(mp * t) * std::cos(t); };
        double a = pi / mp, b = 2.0 * pi / mp;
        double fa = f(a);
        for (int it = 0; it < 200 && b - a > 1e-17; ++it) {
            const double c = 0.5 * (a + b);
            const double fc = f(c);
            if ((fc < 0.0) == (fa < 0.0)) {
                a = c;
                fa = fc;
            } else {
                b = c;
            }
        }
        const double t = 0.5 * (a + b);
        const double sh = std::sin(0.5 * t);
        return sh * sh;
    }

    // The x <= x_1 (first root) with P_m(x) = y; P_m is decreasing there. For y < 0 the
    // reference extends the inverse by the first root (LanczosCpoly.h:429-432).
    static double inverse(long m, double y) {
        const double pi = 3.14159265358979323846;
        const double s1 = std::sin(0.5 * pi / (double)(m + 1));
        const double x1 = s1 * s1;
        if (y < 0.0) return x1;
        double a, b = x1;
        if (y <= 1.0) {
            a = 0.0;
        } else {
            a = -1e-8;
            for (int it = 0; it < 400 && pm(m, a) < y; ++it) a *= 2.0;
        }
        for (int it = 0; it < 300; ++it) {
            const double c = 0.5 * (a + b);
            if (c <= a || c >= b) break;
            if (pm(m, c) > y) a = c; else b = c;
        }
        return 0.5 * (a + b);
    }

    double xstar(long m) {
        if (m <= 0) return 1.0;
        if (m == 1) return 0.3;
        cache(m);
        return xs_[m];
    }
    double upper_xstar(long m) {
        if (m <= 0) return 1.0;
        if (m == 1) return 0.6;
        if (m == 2) return (1.0 - xstar(2) + 0.6) / 2.0;
        const double pi = 3.14159265358979323846;
        return (std::cos(2.0 / ((double)m + 1.0) * pi) + 1.0) * 0.5;
    }
    double ratio(long m) { return xstar(m) / upper_xstar(m); }

    // getStarDegreeAndSpectralRadius (LanczosCpoly.h:498-555)
    void star_degree_and_bound(double shift, double lambdaBound, double lambdaStar, long degMax, long& starDegree,
                               double& starBound) {
        const double lss = lambdaStar + shift;
        double r = ratio(1);
        if (r * (lambdaBound + shift) < lss) {
            starDegree = 1;
            starBound = lss / r - shift;
            return;
        }
        long mb = 2;
        while (mb < degMax) {
            r = ratio(mb);
            if (r * (lambdaBound + shift) < lss) break;
            ++mb;
        }
        if (mb >= degMax) {
            starDegree = degMax;
            starBound = lambdaBound;
            return;
        }
        starDegree = mb;
        starBound = lss / ratio(mb) - shift;
    }

    // Recurrence coefficients of LanczosCpolyOperatorLMCuda::apply (:206-209), in the product
    // form used by the kernels: a = gamma2*gamma1 = -4/rhoB, b = gamma2 = 2 - 4*shift/rhoB.
    void coefficients(long m, double lambdaMax, double shift, double& a, double& b) {
        const double ux = upper_xstar(m);
        const double rhoB = lambdaMax / ux + shift / ux;
        a = -4.0 / rhoB;
        b = 2.0 - (4.0 * shift) / rhoB;
    }

private:
    void cache(long m) {
        if ((long)xs_.size() <= m) xs_.resize(m + 1, -1.0);
        if (xs_[m] < 0.0) {
            const double xp = first_extremum(m);
            const double yp = pm(m, xp);
            xs_[m] = inverse(m, -yp);
        }
    }
    std::vector<double> xs_;
};

}  // namespace rcb
