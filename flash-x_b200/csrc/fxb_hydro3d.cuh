// fxb_hydro3d.cuh -- fused 3-D unsplit hydro step (declarations).
#pragma once
#include "fxb_device.cuh"

namespace fxb {
struct Args3D {
    const double *in;
    double *out;
    long vstride;
    int nx, ny, nz;
    int bc[6];
    double dx, dy, dz;
    double dt_arg;
    const double *dtv;
    double gam1inv, ggprodinv;
    DevParams prm;
    unsigned long long *rate_max;
    int *err;
};
} // namespace fxb

namespace fxb {
// 3-D tile extents (cells per CTA along x, y, z)
constexpr int T3X = 16, T3Y = 8, T3Z = 8;
} // namespace fxb
