// Host-only parts of the C ABI: building and evaluating the spatial kernel lookup
// table.  No GPU is touched here, so these run on any machine that loads the
// library.
#include <cmath>

#include "covidsim_b200.h"

namespace {

// KernelStruct::* (src/Kernels.cpp:68-106), evaluated at squared distance r2.
double kernel_value(int type, double scale, double shape, double p3, double p4, double r2)
{
    double t, d;
    switch (type) {
    case 1: return std::exp(-std::sqrt(r2) / scale);
    case 2:
        t = -shape * std::log(std::sqrt(r2) / scale + 1.0);
        return (t < -690.0) ? 0.0 : std::exp(t);
    case 3: return std::exp(-r2 / (scale * scale));
    case 4: return (r2 > scale * scale) ? 0.0 : 1.0;
    case 5:
        t = 0.5 * shape * std::log(r2 / (scale * scale));
        return (t > 690.0) ? 0.0 : (1.0 / (std::exp(t) + 1.0));
    case 6:
        t = std::log(std::sqrt(r2) / scale + 1.0);
        return (t < -690.0) ? 0.0 : (std::exp(-shape * t) + p3 * std::exp(-p4 * t)) / (1.0 + p3);
    case 7:
        d = std::sqrt(r2);
        t = -shape * std::log(d / scale + 1.0);
        return (t < -690.0) ? 0.0 : std::exp(t - std::pow(d / p3, p4));
    default: return -1.0;
    }
}

}  // namespace

extern "C" int cs_build_kernel_table(int kernel_type, double scale, double shape, double p3, double p4,
                                     double longest_d2, int size, int expansion, double* lookup_out,
                                     double* hi_res_out, double* delta_out)
{
    // KernelLookup::setup + KernelLookup::init(1.0, kernel) (src/Kernels.cpp:8-46)
    if (kernel_type < 1 || kernel_type > 7 || size < 2 || expansion < 1 || !lookup_out || !hi_res_out || !delta_out)
        return CS_E_ARG;
    if (!(longest_d2 > 0)) return CS_E_ARG;
    const double delta = longest_d2 / size;
    for (int i = 0; i <= size; i++) {
        lookup_out[i] = kernel_value(kernel_type, scale, shape, p3, p4, i * delta) / 1.0;
        hi_res_out[i] = kernel_value(kernel_type, scale, shape, p3, p4, i * delta / expansion) / 1.0;
    }
    *delta_out = delta;
    return CS_OK;
}

extern "C" double cs_kernel_num(const double* lookup, const double* hi_res, int size, int expansion, double delta,
                                double r2)
{
    // KernelLookup::num (src/Kernels.cpp:108-129); NaN for a distance past the table,
    // where the reference stops with "r too large in NumKernel".
    double t = r2 / delta;
    if (t > size) return std::nan("");
    double s = t * expansion;
    if (s < size) {
        t = s - std::floor(s);
        t = (1.0 - t) * hi_res[(int)s] + t * hi_res[(int)(s + 1.0)];
    } else {
        int i0 = (int)t, i1 = (int)(t + 1.0);
        if (i1 > size) i1 = size;
        s = t - std::floor(t);
        t = (1.0 - s) * lookup[i0] + s * lookup[i1];
    }
    return t;
}
