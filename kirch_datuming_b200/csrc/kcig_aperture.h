// Aperture weight of one leg (source or receiver) at one image point,
// shared by the table-driven and the surrogate-driven leg-field kernels.
#pragma once

namespace kcig {

// kirchmig2d_cig.cpp:226-269: raised-cosine aperture legs (cos(pi x) as cospi,
// which needs no large-argument reduction), max-combined with
// the shallow floor disk.  Evaluated once per (position, image point) instead
// of once per pair: the value depends only on this leg.
__device__ __forceinline__ double leg_cone(double leg, double aper, double band)
{
    if (!isfinite(leg)) return 0.0;
    if (band <= 0.0) return (leg <= aper) ? 1.0 : 0.0;
    const double inner = aper - band;
    if (leg <= inner) return 1.0;
    if (leg >= aper) return 0.0;
    return 0.5 * (1.0 + cospi((leg - inner) / band));
}

__device__ __forceinline__ double leg_floor(double d, double rmin, double rt)
{
    if (rmin <= 0.0) return 0.0;
    if (rt <= 0.0) return (d <= rmin) ? 1.0 : 0.0;
    const double inner = rmin - rt;
    if (inner <= 0.0) {
        if (d >= rmin) return 0.0;
        return 0.5 * (1.0 + cospi(d / rmin));
    }
    if (d <= inner) return 1.0;
    if (d >= rmin) return 0.0;
    return 0.5 * (1.0 + cospi((d - inner) / rt));
}

// the leg weight of :1221-1263 for a leg at surface position `pos` and the
// image point (iz, ix): cone of half-angle `aper` (degrees, cosine band
// `aper_taper`) max-combined with the floor disk (rmin, rtaper)
__device__ __forceinline__ double leg_aperture_weight(double pos, int iz, int ix, double dz, double x0, double dx,
                                                      double aper, double aper_taper, double rmin, double rtaper)
{
    const double zdist = fmax(fabs((double)iz * dz), fmax(1.0e-12, 1.0e-6 * fabs(dz)));
    const double ximg = x0 + (double)ix * dx;
    const double d = fabs(pos - ximg);
    const double legdeg = atan(d / zdist) * 180.0 / 3.14159265358979323846;
    return fmax(leg_cone(legdeg, aper, aper_taper), leg_floor(d, rmin, rtaper));
}

}  // namespace kcig
