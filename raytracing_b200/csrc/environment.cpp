// The environment map's sampling tables, built on the host in double (the reference's environment_table.cu:81-226,
// whose method this follows: cells of exact solid angle, density Y/S per steradian, and Vose's alias table).
//
// A cell c of row j covers the solid angle (2 pi / W)(cos theta_j - cos theta_{j+1}); its weight is its Rec. 709
// luminance times that, and S is the sum of the weights. A sample picks a cell with chance weight/S from the alias
// table, then a direction uniform over the cell's solid angle, so its density is Y/S, stored in the texel.
//
// The alias table has P = 2^k bins (k >= 1, padded with empty bins), so the device picks a bin from the top k bits of
// one random number. Each bin keeps its own cell with the chance q (a coin on the 2^-24 grid, the granularity of the
// device's uniform numbers) and gives the rest to its alias. The coins are rounded to that grid with error diffusion
// (the running rounding error stays within half a step), and every cell with light keeps at least one step, so it can
// be drawn.
#include <algorithm>
#include <bit>
#include <cmath>
#include <numbers>

#include "host.h"

namespace rtb
{
namespace
{
double luminance(const float* rgb) { return 0.2126 * rgb[0] + 0.7152 * rgb[1] + 0.0722 * rgb[2]; }

constexpr double coin_grid = 16777216.0; // 2^24

// A cell's share of its bin, rounded to the coin grid with error diffusion
double round_coin(double share, double& drift)
{
    if (share == 0)
    {
        return 0;
    }
    const double exact = share * coin_grid;
    double steps = std::floor(exact);
    if (steps == 0 || drift + (steps - exact) < -0.5)
    {
        steps += 1;
    }
    drift += steps - exact;
    return steps / coin_grid;
}

// Vose's method: bins of share below 1 keep it as their coin and take the rest from a bin of share >= 1, which gives
// up exactly 1 - q (exact in double on the coin grid) and is reclassified; the bins left over get q = 1
std::vector<alias_bin> make_alias(std::vector<double> share)
{
    const size_t n = share.size();
    std::vector<alias_bin> bins(n);
    std::vector<uint32_t> below;
    std::vector<uint32_t> above;
    below.reserve(n);
    above.reserve(n);
    for (uint32_t c = 0; c < n; ++c)
    {
        (share[c] < 1 ? below : above).push_back(c);
    }
    double drift = 0;
    while (!below.empty() && !above.empty())
    {
        const uint32_t small = below.back();
        below.pop_back();
        const uint32_t large = above.back();
        above.pop_back();
        const double q = round_coin(share[small], drift);
        bins[small] = {static_cast<float>(q), static_cast<int32_t>(large)};
        share[large] -= 1 - q;
        (share[large] < 1 ? below : above).push_back(large);
    }
    for (const uint32_t c : above)
    {
        bins[c] = {1.0f, static_cast<int32_t>(c)};
    }
    for (const uint32_t c : below)
    {
        bins[c] = {1.0f, static_cast<int32_t>(c)};
    }
    return bins;
}
} // namespace

environment_tables build_environment(const rt_environment_desc& env)
{
    environment_tables t;
    t.width = env.image.width;
    t.height = env.image.height;
    const size_t cells = static_cast<size_t>(t.width) * static_cast<size_t>(t.height);
    std::vector<double> cosines(static_cast<size_t>(t.height) + 1);
    for (int j = 0; j <= t.height; ++j)
    {
        cosines[static_cast<size_t>(j)] = std::cos(std::numbers::pi * j / t.height);
    }
    cosines.front() = 1;
    cosines.back() = -1;
    const auto omega = [&](int j) {
        return 2 * std::numbers::pi / t.width * (cosines[static_cast<size_t>(j)] - cosines[static_cast<size_t>(j) + 1]);
    };
    double total = 0;
    for (int j = 0; j < t.height; ++j)
    {
        double row = 0;
        for (int i = 0; i < t.width; ++i)
        {
            row += luminance(env.image.rgb + 3 * (static_cast<size_t>(j) * t.width + i));
        }
        total += row * omega(j);
    }
    t.total = total;
    for (const double c : cosines)
    {
        t.row_cos.push_back(static_cast<float>(c));
    }
    t.texels.resize(cells);
    for (size_t k = 0; k < cells; ++k)
    {
        const float* rgb = env.image.rgb + 3 * k;
        t.texels[k] = {rgb[0], rgb[1], rgb[2], total > 0 ? static_cast<float>(luminance(rgb) / total) : 0.0f};
    }
    if (total == 0)
    {
        return t; // a black map: nothing to sample
    }
    t.log2_bins = std::max(1, static_cast<int>(std::bit_width(cells - 1)));
    const size_t bins = size_t{1} << t.log2_bins;
    std::vector<double> share(bins, 0.0);
    for (int j = 0; j < t.height; ++j)
    {
        const double o = omega(j);
        for (int i = 0; i < t.width; ++i)
        {
            const size_t c = static_cast<size_t>(j) * t.width + i;
            share[c] = luminance(env.image.rgb + 3 * c) * o * static_cast<double>(bins) / total;
        }
    }
    t.bins = make_alias(std::move(share));
    return t;
}
} // namespace rtb
