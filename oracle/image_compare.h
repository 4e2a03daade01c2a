// TEST INFRASTRUCTURE — ImageCompare, the reference's statistical oracle, restated from src/image_compare.cpp (the
// program is a C++23 module user that GCC cannot build). Are two renders the same picture up to Monte Carlo noise?
// Four checks on d = B - A (image_compare.cpp:1-23): the whole image's mean per channel, Stouffer's sum over 32x32
// tiles, the largest tile, and the count of tiles with |z| > 3, each at a false-alarm rate of 1/400; plus the sign
// test that warns about noise of different shapes.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <numbers>
#include <vector>

namespace oracle
{
// image_compare.cpp:36-67 running_stats: Welford's one-pass mean and spread
class running_stats
{
public:
    void add(double x)
    {
        ++count_;
        const double delta = x - mean_;
        mean_ += delta / static_cast<double>(count_);
        squared_deviations_ += delta * (x - mean_);
        sum_of_squares_ += x * x;
    }
    int64_t count() const { return count_; }
    double mean() const { return mean_; }
    double variance() const { return count_ > 1 ? squared_deviations_ / static_cast<double>(count_ - 1) : 0.0; }
    double rms() const { return count_ > 0 ? std::sqrt(sum_of_squares_ / static_cast<double>(count_)) : 0.0; }

private:
    int64_t count_ = 0;
    double mean_ = 0;
    double squared_deviations_ = 0;
    double sum_of_squares_ = 0;
};

inline double normal_tail(double z) { return std::erfc(z / std::numbers::sqrt2); } // image_compare.cpp:71-74

inline double normal_quantile(double p) // image_compare.cpp:78-98: bisection over [0, 40]
{
    if (!(p > 0))
    {
        return std::numeric_limits<double>::infinity();
    }
    double low = 0;
    double high = 40;
    for (int i = 0; i < 60; ++i)
    {
        const double middle = (low + high) / 2;
        if (normal_tail(middle) > p)
        {
            low = middle;
        }
        else
        {
            high = middle;
        }
    }
    return (low + high) / 2;
}

// image_compare.cpp:103-152: I_x(a, b) by the continued fraction (Numerical Recipes 6.4, modified Lentz)
inline double incomplete_beta(double a, double b, double x)
{
    if (x <= 0)
    {
        return 0;
    }
    if (x >= 1)
    {
        return 1;
    }
    if (x > (a + 1) / (a + b + 2))
    {
        return 1 - incomplete_beta(b, a, 1 - x);
    }
    const double log_front = a * std::log(x) + b * std::log1p(-x) + std::lgamma(a + b) - std::lgamma(a) - std::lgamma(b);
    constexpr double tiny = 1e-300;
    const auto nonzero = [](double v) { return std::fabs(v) < tiny ? tiny : v; };
    double c = 1;
    double d = 1 / nonzero(1 - (a + b) * x / (a + 1));
    double fraction = d;
    for (int m = 1; m <= 100000; ++m)
    {
        const std::array<double, 2> pair{m * (b - m) * x / ((a + 2 * m - 1) * (a + 2 * m)),
                                         -(a + m) * (a + b + m) * x / ((a + 2 * m) * (a + 2 * m + 1))};
        for (const double k : pair)
        {
            d = 1 / nonzero(1 + k * d);
            c = nonzero(1 + k / c);
            fraction *= c * d;
        }
        if (std::fabs(c * d - 1) < 1e-15)
        {
            break;
        }
    }
    return std::exp(log_front) * fraction / a;
}

// image_compare.cpp:157-166: the z exactly as rare as Student's t with df degrees of freedom
inline double normal_equivalent(double t, double df)
{
    const double p = incomplete_beta(df / 2, 0.5, df / (df + t * t));
    if (p > 0 || std::isinf(t))
    {
        return std::copysign(normal_quantile(p), t);
    }
    return std::copysign(std::sqrt(df * std::log1p(t * t / df)), t);
}

// image_compare.cpp:171-187: P(K >= k) for a binomial K
inline double binomial_tail(int n, double q, int k)
{
    double sum = 0;
    for (int j = std::max(k, 0); j <= n; ++j)
    {
        const double log_term = std::lgamma(n + 1.0) - std::lgamma(j + 1.0) - std::lgamma(n - j + 1.0) +
                                j * std::log(q) + (n - j) * std::log1p(-q);
        const double term = std::exp(log_term);
        sum += term;
        if (j > n * q && term < 1e-17 * sum)
        {
            break;
        }
    }
    return sum;
}

constexpr double rounding_margin = 1e-6;                       // image_compare.cpp:198
constexpr double sign_test_threshold = 1000 * rounding_margin;  // image_compare.cpp:272
constexpr int default_tile_size = 32;
constexpr double false_alarm_rate_per_check = 1.0 / 400;       // image_compare.cpp:408
constexpr double tile_z_counted = 3;
constexpr double tile_z_clamp = 40;
constexpr double sign_test_beyond_chance = 5;
constexpr double sign_test_to_all_tiles = 3;

struct mean_test
{
    double mean = 0;
    double standard_error = 0;
    double z = 0;
};

// image_compare.cpp:246-260 test_mean: z of the mean beyond the rounding margin, Student's t turned into z
inline mean_test test_mean(const running_stats& d, double level)
{
    const double standard_error = std::sqrt(d.variance() / static_cast<double>(d.count()));
    const double beyond_rounding = std::fabs(d.mean()) - rounding_margin * level;
    double z = 0;
    if (beyond_rounding > 0)
    {
        const double t = standard_error > 0 ? beyond_rounding / standard_error : std::numeric_limits<double>::infinity();
        z = std::copysign(normal_equivalent(t, static_cast<double>(d.count() - 1)), d.mean());
    }
    return {d.mean(), standard_error, z};
}

struct tile
{
    int x0 = 0, y0 = 0, x1 = 0, y1 = 0;
    running_stats d;
    double level_sum = 0;
    mean_test test;
    bool has_spread() const { return d.count() >= 2; }
    bool identical() const { return d.rms() == 0; }
};

struct thresholds
{
    double whole_image = 0;
    double all_tiles = 0;
    double largest_tile = 0;
    int tiles_over_3 = 0;
};

// image_compare.cpp:442-458 alarm_thresholds
inline thresholds alarm_thresholds(int tested_tiles)
{
    thresholds r{normal_quantile(false_alarm_rate_per_check / 4), normal_quantile(false_alarm_rate_per_check), 0, 0};
    if (tested_tiles > 0)
    {
        r.largest_tile = normal_quantile(false_alarm_rate_per_check / tested_tiles);
        const double q = normal_tail(tile_z_counted);
        r.tiles_over_3 = std::max(1, static_cast<int>(tested_tiles * q));
        while (binomial_tail(tested_tiles, q, r.tiles_over_3) > false_alarm_rate_per_check)
        {
            ++r.tiles_over_3;
        }
    }
    return r;
}

// Everything ImageCompare prints, as numbers; verdict 0 consistent, 1 different, 2 an error (image_compare.cpp:786-873)
struct compare_result
{
    int verdict = 2;
    double mean_a = 0, mean_b = 0;          // mean radiance of each image
    double channel_mean[4] = {};            // red, green, blue, average of d
    double channel_se[4] = {};
    double channel_z[4] = {};
    double channel_level[4] = {};
    double channel_rms[4] = {};
    double whole_image_z = 0;               // the largest |z| of the 4 rows
    double all_tiles_z = 0;                 // Stouffer's sum / sqrt(T)
    double largest_tile_z = 0;
    int tiles_over_3 = 0;
    int tested_tiles = 0;
    int identical_tiles = 0;
    double threshold_whole_image = 0, threshold_all_tiles = 0, threshold_largest_tile = 0;
    int threshold_tiles_over_3 = 0;
    int failed_whole_image = 0, failed_all_tiles = 0, failed_largest_tile = 0, failed_tile_count = 0;
    int64_t sign_b_brighter = 0, sign_a_brighter = 0;
    double sign_z = 0;
    int noise_shapes_differ = 0;
    int non_finite = 0;
    int largest_tile_x0 = 0, largest_tile_y0 = 0;
};

struct tile_summary
{
    int tested = 0;
    int identical = 0;
    double all_tiles_z = 0;
    int over_3 = 0;
    const tile* largest = nullptr;
};

inline tile_summary summarize(const std::vector<tile>& tiles) // image_compare.cpp:470-500
{
    tile_summary s;
    double z_sum = 0;
    for (const tile& t : tiles)
    {
        if (!t.has_spread())
        {
            continue;
        }
        if (t.identical())
        {
            ++s.identical;
            continue;
        }
        ++s.tested;
        z_sum += std::clamp(t.test.z, -tile_z_clamp, tile_z_clamp);
        if (std::fabs(t.test.z) > tile_z_counted)
        {
            ++s.over_3;
        }
        if (!s.largest || std::fabs(t.test.z) > std::fabs(s.largest->test.z))
        {
            s.largest = &t;
        }
    }
    s.all_tiles_z = s.tested > 0 ? z_sum / std::sqrt(s.tested) : 0.0;
    return s;
}

// image_compare.cpp:333-399 compare + the checks of main. a and b: width*height*3 linear values, rows from the top.
inline compare_result image_compare(const float* a, const float* b, int width, int height, int tile_size)
{
    compare_result out;
    const int64_t n = static_cast<int64_t>(width) * height;
    for (int64_t i = 0; i < 3 * n; ++i)
    {
        if (!std::isfinite(a[i]) || !std::isfinite(b[i]))
        {
            ++out.non_finite;
        }
    }
    if (out.non_finite > 0 || n < 2 || tile_size < 2)
    {
        out.verdict = 2;
        return out;
    }
    double sum_a = 0, sum_b = 0;
    for (int64_t i = 0; i < n; ++i)
    {
        sum_a += (static_cast<double>(a[3 * i]) + a[3 * i + 1] + a[3 * i + 2]) / 3;
        sum_b += (static_cast<double>(b[3 * i]) + b[3 * i + 1] + b[3 * i + 2]) / 3;
    }
    out.mean_a = sum_a / static_cast<double>(n);
    out.mean_b = sum_b / static_cast<double>(n);

    const auto run = [&](int ts, std::vector<tile>& tiles, std::array<running_stats, 4>& d,
                         std::array<double, 4>& level_sum, int64_t& b_brighter, int64_t& a_brighter) {
        const int tiles_x = (width - 1) / ts + 1;
        const int tiles_y = (height - 1) / ts + 1;
        for (int ty = 0; ty < tiles_y; ++ty)
        {
            for (int tx = 0; tx < tiles_x; ++tx)
            {
                tile t;
                t.x0 = tx * ts;
                t.y0 = ty * ts;
                t.x1 = std::min((tx + 1) * ts, width);
                t.y1 = std::min((ty + 1) * ts, height);
                tiles.push_back(t);
            }
        }
        for (int y = 0; y < height; ++y)
        {
            for (int x = 0; x < width; ++x)
            {
                const int64_t p = static_cast<int64_t>(y) * width + x;
                const double ar = a[3 * p], ag = a[3 * p + 1], ab = a[3 * p + 2];
                const double br = b[3 * p], bg = b[3 * p + 1], bb = b[3 * p + 2];
                const double dr = br - ar, dg = bg - ag, db = bb - ab;
                const double lr = (std::fabs(ar) + std::fabs(br)) / 2;
                const double lg = (std::fabs(ag) + std::fabs(bg)) / 2;
                const double lb = (std::fabs(ab) + std::fabs(bb)) / 2;
                const std::array<double, 4> differences{dr, dg, db, (dr + dg + db) / 3};
                const std::array<double, 4> levels{lr, lg, lb, (lr + lg + lb) / 3};
                for (size_t c = 0; c < 4; ++c)
                {
                    d[c].add(differences[c]);
                    level_sum[c] += levels[c];
                }
                const double threshold = sign_test_threshold * levels[3];
                if (differences[3] > threshold)
                {
                    ++b_brighter;
                }
                else if (differences[3] < -threshold)
                {
                    ++a_brighter;
                }
                tile& t = tiles[static_cast<size_t>(y / ts) * static_cast<size_t>(tiles_x) + static_cast<size_t>(x / ts)];
                t.d.add(differences[3]);
                t.level_sum += levels[3];
            }
        }
        for (tile& t : tiles)
        {
            if (t.has_spread())
            {
                t.test = test_mean(t.d, t.level_sum / static_cast<double>(t.d.count()));
            }
        }
    };

    std::vector<tile> tiles;
    std::array<running_stats, 4> d;
    std::array<double, 4> level_sum{};
    run(tile_size, tiles, d, level_sum, out.sign_b_brighter, out.sign_a_brighter);
    bool all_identical = true;
    for (size_t c = 0; c < 4; ++c)
    {
        out.channel_level[c] = level_sum[c] / static_cast<double>(n);
        const mean_test t = test_mean(d[c], out.channel_level[c]);
        out.channel_mean[c] = t.mean;
        out.channel_se[c] = t.standard_error;
        out.channel_z[c] = t.z;
        out.channel_rms[c] = d[c].rms();
        all_identical = all_identical && d[c].rms() == 0;
        out.whole_image_z = std::max(out.whole_image_z, std::fabs(t.z));
    }
    if (all_identical)
    {
        out.verdict = 2; // the same random numbers: nothing to compare
        return out;
    }
    const tile_summary summary = summarize(tiles);
    const thresholds limits = alarm_thresholds(summary.tested);
    out.tested_tiles = summary.tested;
    out.identical_tiles = summary.identical;
    out.all_tiles_z = summary.all_tiles_z;
    out.tiles_over_3 = summary.over_3;
    out.threshold_whole_image = limits.whole_image;
    out.threshold_all_tiles = limits.all_tiles;
    out.threshold_largest_tile = limits.largest_tile;
    out.threshold_tiles_over_3 = limits.tiles_over_3;
    out.failed_whole_image = out.whole_image_z > limits.whole_image;
    if (summary.largest)
    {
        out.largest_tile_z = std::fabs(summary.largest->test.z);
        out.largest_tile_x0 = summary.largest->x0;
        out.largest_tile_y0 = summary.largest->y0;
        out.failed_all_tiles = std::fabs(summary.all_tiles_z) > limits.all_tiles;
        out.failed_largest_tile = out.largest_tile_z > limits.largest_tile;
        out.failed_tile_count = summary.over_3 >= limits.tiles_over_3;
    }
    const int64_t differing = out.sign_b_brighter + out.sign_a_brighter;
    out.sign_z = differing > 0 ? static_cast<double>(out.sign_b_brighter - out.sign_a_brighter) /
                                     std::sqrt(static_cast<double>(differing))
                               : 0.0;
    double all_tiles_z = summary.all_tiles_z;
    if (tile_size != default_tile_size)
    {
        std::vector<tile> small;
        std::array<running_stats, 4> d2;
        std::array<double, 4> l2{};
        int64_t bb = 0, aa = 0;
        run(default_tile_size, small, d2, l2, bb, aa);
        all_tiles_z = summarize(small).all_tiles_z;
    }
    const double same_way = out.sign_z > 0 ? all_tiles_z : -all_tiles_z;
    out.noise_shapes_differ =
        std::fabs(out.sign_z) > sign_test_beyond_chance && same_way < std::fabs(out.sign_z) / sign_test_to_all_tiles;
    const bool failed = out.failed_whole_image || out.failed_all_tiles || out.failed_largest_tile || out.failed_tile_count;
    out.verdict = failed ? 1 : 0;
    return out;
}
} // namespace oracle
