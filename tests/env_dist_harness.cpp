// Test harness: the library's environment-sampling tables (env_dist.hpp)
// against the oracle's restatement (oracle.hpp, Scene::build_env_distribution)
// for the environment read from argv[1] (u32 w, u32 h, w*h*3 floats).
// Prints "ok <sum of pdf * solid angle>" when every table is bit-identical.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "env_dist.hpp"
#include "../oracle/oracle.hpp"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    uint32_t wh[2];
    if (std::fread(wh, 4, 2, f) != 2) return 2;
    std::vector<float> rgb((size_t)wh[0] * wh[1] * 3);
    if (std::fread(rgb.data(), 4, rgb.size(), f) != rgb.size()) return 2;
    std::fclose(f);
    const cupbr_b200::EnvDistribution d = cupbr_b200::build_env_distribution(rgb.data(), wh[0], wh[1]);
    oracle::Scene<float> sc;
    sc.env_w = wh[0];
    sc.env_h = wh[1];
    for (size_t i = 0; i < (size_t)wh[0] * wh[1]; ++i) sc.env.push_back(oracle::V3<float>(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]));
    sc.build_env_distribution();
    auto same = [](const std::vector<float>& a, const std::vector<float>& b) {
        return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(float)) == 0;
    };
    if (d.cw != sc.env_cw || d.ch != sc.env_ch || !same(d.marg, sc.env_marg) || !same(d.cond, sc.env_cond) ||
        !same(d.pdf, sc.env_pdf) || !same(d.cosb, sc.env_cosb)) {
        std::printf("mismatch\n");
        return 1;
    }
    // the density integrates to one over the sphere: sum of pdf * cell solid angle
    const double pi = 3.14159265358979323846;
    double total = 0.0;
    for (uint32_t y = 0; y < d.ch; ++y) {
        const double om = (2.0 * pi / d.cw) * (std::cos(pi * y / d.ch) - std::cos(pi * (y + 1) / d.ch));
        for (uint32_t x = 0; x < d.cw; ++x) total += (double)d.pdf[(size_t)y * d.cw + x] * om;
    }
    std::printf("ok %.9f\n", total);
    return 0;
}
