// Importance-sampling tables of the environment map for the physical
// estimator (MIS between environment sampling and BSDF sampling).
//
// The reference looks the environment up with the nearest texel of the
// direction's lat-long coordinates (Tracing::direction2UV,
// lib/src/Core/TracingDetail.h:185-196): x = (w-1)*phi, y = (h-1)*theta/pi,
// truncated.  So radiance is constant over the cells of a cw x ch grid
// (cw = w-1, ch = h-1; a 1-texel axis counts as one cell), cell (x, y)
// spanning phi in [x, x+1)/cw and theta in [y, y+1)*pi/ch with texel (x, y)'s
// value.  A cell is chosen with probability proportional to its mean
// channel value times its solid angle, and a direction uniformly inside its
// solid angle, so the density per solid angle is lum(cell) / sum over cells
// of lum * solid angle: a constant per cell, stored in `pdf`.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

namespace cupbr_b200 {

struct EnvDistribution {
    uint32_t cw = 0, ch = 0;
    std::vector<float> marg;  // ch: CDF over rows (last entry 1)
    std::vector<float> cond;  // ch * cw: CDF over the cells of each row (last entry of a row 1)
    std::vector<float> pdf;   // ch * cw: density per solid angle of a direction in the cell
    std::vector<float> cosb;  // ch + 1: cos(theta) at the row boundaries, cos(pi * y / ch)
};

// rgb: w * h texels of 3 floats, row-major (row y = theta index).
inline EnvDistribution build_env_distribution(const float* rgb, uint32_t w, uint32_t h) {
    EnvDistribution D;
    if (w == 0 || h == 0) return D;
    const uint32_t cw = w > 1 ? w - 1 : 1, ch = h > 1 ? h - 1 : 1;
    D.cw = cw;
    D.ch = ch;
    D.marg.resize(ch);
    D.cond.resize((size_t)cw * ch);
    D.pdf.resize((size_t)cw * ch);
    D.cosb.resize(ch + 1);
    const double pi = 3.14159265358979323846;
    for (uint32_t y = 0; y <= ch; ++y) D.cosb[y] = (float)std::cos(pi * (double)y / (double)ch);
    D.cosb[0] = 1.0f;
    D.cosb[ch] = -1.0f;
    std::vector<double> lum((size_t)cw * ch), row(ch), omega(ch);
    double total = 0.0;
    for (uint32_t y = 0; y < ch; ++y) {
        // solid angle of a cell of row y
        omega[y] = (2.0 * pi / (double)cw) * (std::cos(pi * y / (double)ch) - std::cos(pi * (y + 1) / (double)ch));
        double r = 0.0;
        for (uint32_t x = 0; x < cw; ++x) {
            const float* t = rgb + 3 * ((size_t)x + (size_t)y * w);
            double l = ((double)t[0] + (double)t[1] + (double)t[2]) / 3.0;
            if (!(l > 0.0) || !std::isfinite(l)) l = 0.0;
            lum[(size_t)y * cw + x] = l;
            r += l * omega[y];
        }
        row[y] = r;
        total += r;
    }
    double acc = 0.0;
    for (uint32_t y = 0; y < ch; ++y) {
        acc += row[y];
        D.marg[y] = total > 0.0 ? (float)(acc / total) : (float)((double)(y + 1) / (double)ch);
        double a = 0.0;
        for (uint32_t x = 0; x < cw; ++x) {
            const size_t i = (size_t)y * cw + x;
            a += lum[i] * omega[y];
            D.cond[i] = row[y] > 0.0 ? (float)(a / row[y]) : (float)((double)(x + 1) / (double)cw);
            D.pdf[i] = total > 0.0 ? (float)(lum[i] / total) : 0.0f;
        }
        D.cond[(size_t)y * cw + cw - 1] = 1.0f;
    }
    D.marg[ch - 1] = 1.0f;
    return D;
}

}  // namespace cupbr_b200
