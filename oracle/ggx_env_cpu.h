// TEST INFRASTRUCTURE — the oracle's GGX lobes and environment map, in double.
//
// Restated from the equations the reference cites (src/gpu/ggx.cuh:1-325: Walter et al. 2007, Heitz 2014 and 2018,
// Dupuy & Benyoub 2023, Turquin 2019, Ashikhmin & Shirley 2000; src/gpu/environment.cuh, background.cuh and
// environment_table.cu: the equirectangular +y-up map, cells of exact solid angle, Vose's alias table with coins on
// the 2^-24 grid). The reference has these on the GPU only; here they run on the CPU renderer of cpu_renderer.h, in
// double, with the CPU's random numbers. Turquin's energy table is computed by this file's own quadrature.
#pragma once

#include <array>
#include <bit>
#include <cmath>
#include <cstdint>
#include <numbers>
#include <thread>
#include <vector>

#include "cpu_renderer.h"

namespace oracle
{
constexpr double min_ggx_alpha = 1e-3; // ggx.cuh:37: below it, the perfect mirror with Schlick's F

inline double smith_a(double c, double alpha2) { return std::sqrt(c * c * (1 - alpha2) + alpha2); }

inline double ggx_d(const vec3& n, const vec3& h, double alpha2) // Walter eq. 33, sin^2 from |n x h|^2
{
    const double c = dot(n, h);
    if (!(c > 0))
    {
        return 0;
    }
    const vec3 s = cross(n, h);
    const double d = alpha2 * c * c + dot(s, s);
    return alpha2 / (std::numbers::pi * d * d);
}

inline color schlick(const color& f0, double cosine)
{
    const double x = std::fmax(0.0, 1 - cosine);
    const double x5 = x * x * x * x * x;
    return {f0.x + (1 - f0.x) * x5, f0.y + (1 - f0.y) * x5, f0.z + (1 - f0.z) * x5};
}

// f * cos(theta_l) and the visible-normal density of l (ggx.cuh:100-126)
inline color ggx_eval(const vec3& n, const vec3& v, const vec3& l, double alpha, const color& f0, double& pdf)
{
    pdf = 0;
    const double cv = dot(n, v);
    const double cl = dot(n, l);
    const vec3 sum = v + l;
    const double len2 = sum.length_squared();
    if (!(cv > 0) || !(cl > 0) || !(len2 > 0))
    {
        return {0, 0, 0};
    }
    const vec3 h = sum / std::sqrt(len2);
    const double alpha2 = alpha * alpha;
    const double d = ggx_d(n, h, alpha2);
    const double av = smith_a(cv, alpha2);
    const double al = smith_a(cl, alpha2);
    pdf = d / (2 * (cv + av));
    return (d * cl / (2 * (cl * av + cv * al))) * schlick(f0, dot(v, h));
}

// A direction by the visible normals, with spherical caps (ggx.cuh:141-200), from two numbers u1 (azimuth), u2
// (height in the cap); false: absorbed. weight = f cos / p (F * G2 / G1), pdf the visible-normal density.
inline bool ggx_sample(const vec3& n, const vec3& v, double alpha, const color& f0, double u1, double u2, vec3& l,
                       color& weight, double& pdf)
{
    const double cv = dot(n, v);
    if (!(cv > 0))
    {
        return false;
    }
    const vec3 vs = unit_vector(alpha * (v - cv * n) + cv * n);
    const double zs = dot(n, vs);
    const double z = (1 - u2) * (1 + zs) - zs;
    const double sin_theta = std::sqrt(std::fmax(0.0, 1 - z * z));
    const double phi = 2 * std::numbers::pi * u1;
    const onb frame{n};
    const vec3 c = frame.transform({sin_theta * std::cos(phi), sin_theta * std::sin(phi), z});
    const vec3 hs = c + vs;
    const double hn = dot(n, hs);
    const vec3 m = alpha * (hs - hn * n) + std::fmax(0.0, hn) * n;
    const double m2 = m.length_squared();
    if (!(m2 > 0))
    {
        return false;
    }
    const vec3 h = m / std::sqrt(m2);
    const double vh = dot(v, h);
    l = (2 * vh) * h - v;
    const double cl = dot(n, l);
    if (!(cl > 0) || !(vh > 0))
    {
        return false;
    }
    const double alpha2 = alpha * alpha;
    const double av = smith_a(cv, alpha2);
    const double al = smith_a(cl, alpha2);
    weight = (cl * (cv + av) / (cl * av + cv * al)) * schlick(f0, vh);
    pdf = ggx_d(n, h, alpha2) / (2 * (cv + av));
    return true;
}

// Turquin's table: E_ss(mu, r) of a white conductor (F = 1), nodes sqrt(mu) = i/31 and r = j/31 (ggx.cuh:202-236),
// row 0 and column 0 equal to 1. E = integral over the visible normals of G2/G1, computed here on the sampling's own
// parameters: the azimuth by the trapezoidal rule (periodic, so spectrally accurate), and for each azimuth the valid
// heights [0, u*] (found by bisection; the light falls below the horizon past u*) by 24-point Gauss-Legendre on
// three sub-intervals.
constexpr int ggx_energy_size = 32;

inline double ggx_energy_quadrature(double mu, double r)
{
    const double alpha = r * r;
    const vec3 n{0, 0, 1};
    const vec3 v{std::sqrt(std::fmax(0.0, 1 - mu * mu)), 0, mu};
    const color white{1, 1, 1};
    static const std::array<double, 24> x = {
        -0.9951872199970213, -0.9747285559713095, -0.9382745520027328, -0.8864155270044011, -0.8200019859739029,
        -0.7401241915785544, -0.6480936519369755, -0.5454214713888396, -0.4337935076260451, -0.3150426796961634,
        -0.1911188674736163, -0.0640568928626056, 0.0640568928626056,  0.1911188674736163,  0.3150426796961634,
        0.4337935076260451,  0.5454214713888396,  0.6480936519369755,  0.7401241915785544,  0.8200019859739029,
        0.8864155270044011,  0.9382745520027328,  0.9747285559713095,  0.9951872199970213};
    static const std::array<double, 24> w = {
        0.0123412297999872, 0.0285313886289337, 0.0442774388174198, 0.0592985849154368, 0.0733464814110803,
        0.0861901615319533, 0.0976186521041139, 0.1074442701159656, 0.1155056680537256, 0.1216704729278034,
        0.1258374563468283, 0.1279381953467522, 0.1279381953467522, 0.1258374563468283, 0.1216704729278034,
        0.1155056680537256, 0.1074442701159656, 0.0976186521041139, 0.0861901615319533, 0.0733464814110803,
        0.0592985849154368, 0.0442774388174198, 0.0285313886289337, 0.0123412297999872};
    const auto value = [&](double u1, double u2, bool& valid) {
        vec3 l;
        color weight;
        double pdf;
        valid = ggx_sample(n, v, alpha, white, u1, u2, l, weight, pdf);
        return valid ? weight.x : 0.0;
    };
    const int azimuths = 256;
    const int scan = 128;
    double total = 0;
    const auto is_valid = [&](double u1, double u2) {
        bool valid;
        value(u1, u2, valid);
        return valid;
    };
    for (int a = 0; a < azimuths; ++a)
    {
        const double u1 = (a + 0.5) / azimuths;
        // The heights where the sample is valid can form several pieces: probe, bisect each change, integrate pieces
        bool inside = is_valid(u1, 0.0);
        double start = 0;
        std::vector<std::pair<double, double>> pieces;
        for (int k = 1; k <= scan; ++k)
        {
            const double u = static_cast<double>(k) / scan;
            const bool now = is_valid(u1, u);
            if (now != inside)
            {
                double lo = static_cast<double>(k - 1) / scan;
                double hi = u;
                for (int it = 0; it < 55; ++it)
                {
                    const double mid = 0.5 * (lo + hi);
                    (is_valid(u1, mid) == inside ? lo : hi) = mid;
                }
                const double edge = 0.5 * (lo + hi);
                if (inside)
                {
                    pieces.emplace_back(start, edge);
                }
                start = edge;
                inside = now;
            }
        }
        if (inside)
        {
            pieces.emplace_back(start, 1.0);
        }
        double line = 0;
        for (const auto& [p0, p1] : pieces)
        {
            for (int part = 0; part < 4; ++part)
            {
                const double a0 = p0 + (p1 - p0) * part / 4;
                const double b0 = p0 + (p1 - p0) * (part + 1) / 4;
                for (size_t k = 0; k < x.size(); ++k)
                {
                    bool valid;
                    const double u2 = 0.5 * (a0 + b0) + 0.5 * (b0 - a0) * x[k];
                    line += 0.5 * (b0 - a0) * w[k] * value(u1, u2, valid);
                }
            }
        }
        total += line;
    }
    return total / azimuths;
}

// Computed once per process (a row per thread), then shared
inline const std::vector<double>& ggx_energy_table()
{
    static const std::vector<double> table = [] {
        std::vector<double> t(ggx_energy_size * ggx_energy_size, 1.0);
        std::vector<std::thread> rows;
        for (int j = 1; j < ggx_energy_size; ++j)
        {
            rows.emplace_back([&t, j] {
                for (int i = 1; i < ggx_energy_size; ++i)
                {
                    const double s = static_cast<double>(i) / (ggx_energy_size - 1);
                    t[static_cast<size_t>(j * ggx_energy_size + i)] =
                        ggx_energy_quadrature(s * s, static_cast<double>(j) / (ggx_energy_size - 1));
                }
            });
        }
        for (std::thread& r : rows)
        {
            r.join();
        }
        return t;
    }();
    return table;
}

inline double ggx_energy(const std::vector<double>& table, double cos_v, double roughness) // bilinear, clamped
{
    constexpr int last = ggx_energy_size - 1;
    const double x = std::sqrt(std::fmin(std::fmax(cos_v, 0.0), 1.0)) * last;
    const double y = std::fmin(std::fmax(roughness, 0.0), 1.0) * last;
    const int i = std::min(static_cast<int>(x), last - 1);
    const int j = std::min(static_cast<int>(y), last - 1);
    const double fx = x - i;
    const double fy = y - j;
    const double* row = table.data() + j * ggx_energy_size + i;
    const double below = (1 - fx) * row[0] + fx * row[1];
    const double above = (1 - fx) * row[ggx_energy_size] + fx * row[ggx_energy_size + 1];
    return (1 - fy) * below + fy * above;
}

inline color ggx_compensation(const std::vector<double>& table, const color& f0, double cos_v, double roughness)
{
    const double e = std::fmin(ggx_energy(table, cos_v, roughness), 1.0);
    const double lost = (1 - e) / e;
    return {1 + f0.x * lost, 1 + f0.y * lost, 1 + f0.z * lost};
}

// The glossy coat (ggx.cuh:238-325): GGX with F0 = 0.04 plus Ashikhmin & Shirley's coupled diffuse base
constexpr double gloss_coat_f0 = 0.04;
inline double gloss_crossing(double c)
{
    const double x = 1 - 0.5 * c;
    return 1 - x * x * x * x * x;
}

inline color gloss_eval(const vec3& n, const vec3& v, const vec3& l, double alpha, const color& rho, double& pdf)
{
    pdf = 0;
    const double cv = dot(n, v);
    const double cl = dot(n, l);
    if (!(cv > 0) || !(cl > 0))
    {
        return {0, 0, 0};
    }
    double coat_pdf;
    const color coat = ggx_eval(n, v, l, alpha, color{gloss_coat_f0, gloss_coat_f0, gloss_coat_f0}, coat_pdf);
    pdf = 0.5 * (coat_pdf + cl / std::numbers::pi);
    const double scale = 28.0 / (23.0 * std::numbers::pi) * (1 - gloss_coat_f0);
    const double base = scale * (gloss_crossing(cl) * gloss_crossing(cv)) * cl;
    return coat + base * rho;
}

// ---- the environment map ----------------------------------------------------------------------------------
struct environment
{
    int width = 0, height = 0;
    double cos_yaw = 1, sin_yaw = 0, scale = 1;
    std::vector<color> texels;       // radiance
    std::vector<double> pdf;          // Y / S per cell
    std::vector<double> row_cos;      // height + 1
    std::vector<double> cell_chance;  // the alias table's chance of each cell (its weight / S), for sampling
    std::vector<double> cell_cdf;     // running sums of cell_chance, for drawing a cell by inversion
    double total = 0;

    bool sampled() const { return total > 0; }

    vec3 to_map(const vec3& d) const { return {cos_yaw * d.x + sin_yaw * d.z, d.y, -sin_yaw * d.x + cos_yaw * d.z}; }
    vec3 from_map(const vec3& d) const { return {cos_yaw * d.x - sin_yaw * d.z, d.y, sin_yaw * d.x + cos_yaw * d.z}; }

    // environment.cuh:36-66: u = 0.5 + atan2(z, x)/(2 pi), t = atan2(sqrt(x^2 + z^2), y)/pi
    void coordinates(const vec3& m, double& u, double& t) const
    {
        u = 0.5 + std::atan2(m.z, m.x) / (2 * std::numbers::pi);
        t = std::atan2(std::sqrt(m.x * m.x + m.z * m.z), m.y) / std::numbers::pi;
    }

    int cell(const vec3& world) const
    {
        double u, t;
        coordinates(to_map(world), u, t);
        const int i = std::clamp(static_cast<int>(u * width), 0, width - 1);
        const int j = std::clamp(static_cast<int>(t * height), 0, height - 1);
        return j * width + i;
    }

    color radiance(const vec3& dir, double& density) const
    {
        const int c = cell(dir);
        density = pdf[static_cast<size_t>(c)];
        return scale * texels[static_cast<size_t>(c)];
    }

    color radiance_filtered(const vec3& dir) const // environment.cuh:110-135: bilinear between texel centres
    {
        double u, t;
        coordinates(to_map(dir), u, t);
        const double x = u * width - 0.5;
        const double y = t * height - 0.5;
        const double x0 = std::floor(x);
        const double y0 = std::floor(y);
        const double fx = x - x0;
        const double fy = y - y0;
        const int i = static_cast<int>(x0);
        const int i0 = i < 0 ? i + width : i;
        const int i1 = i0 + 1 < width ? i0 + 1 : 0;
        const int j = static_cast<int>(y0);
        const int j0 = std::clamp(j, 0, height - 1) * width;
        const int j1 = std::clamp(j + 1, 0, height - 1) * width;
        const auto at = [&](int k) { return texels[static_cast<size_t>(k)]; };
        const color top = at(j0 + i0) + fx * (at(j0 + i1) - at(j0 + i0));
        const color bottom = at(j1 + i0) + fx * (at(j1 + i1) - at(j1 + i0));
        return scale * (top + fy * (bottom - top));
    }

    vec3 cell_direction(int i, int j, double s_theta, double s_phi) const // environment.cuh:73-88
    {
        const double top = row_cos[static_cast<size_t>(j)];
        const double bottom = row_cos[static_cast<size_t>(j) + 1];
        const double cos_theta = top - s_theta * (top - bottom);
        const double sin_theta = std::sqrt(std::fmax(0.0, (1 - cos_theta) * (1 + cos_theta)));
        const double phi = 2 * std::numbers::pi * (i + s_phi) / width - std::numbers::pi;
        return from_map({sin_theta * std::cos(phi), cos_theta, sin_theta * std::sin(phi)});
    }

    // A direction by the map's brightness (background.cuh:77-95): a cell by its chance Y*Omega/S, drawn here by
    // inversion of the running sums (the same distribution as the alias table), then uniform over the cell
    bool sample(rng& g, vec3& wi, color& le, double& density) const
    {
        if (!sampled())
        {
            return false;
        }
        const double xi = g.next();
        const auto it = std::upper_bound(cell_cdf.begin(), cell_cdf.end(), xi * cell_cdf.back());
        int c = static_cast<int>(it - cell_cdf.begin());
        c = std::min(c, width * height - 1);
        const int j = c / width;
        const int i = c - j * width;
        const double s_theta = g.next();
        const double s_phi = g.next();
        wi = cell_direction(i, j, s_theta, s_phi);
        le = radiance(wi, density);
        return density > 0;
    }
};

// environment_table.cu:173-226: rows' cosines cos(pi j / H) with exact ends, S = sum Y * Omega, pdf = Y / S
inline environment make_environment(const rt_environment_desc& d)
{
    environment e;
    e.width = d.image.width;
    e.height = d.image.height;
    const double yaw = d.yaw_degrees * std::numbers::pi / 180;
    e.cos_yaw = std::cos(yaw);
    e.sin_yaw = std::sin(yaw);
    e.scale = d.scale;
    const size_t n = static_cast<size_t>(e.width) * static_cast<size_t>(e.height);
    e.texels.resize(n);
    for (size_t k = 0; k < n; ++k)
    {
        e.texels[k] = {d.image.rgb[3 * k], d.image.rgb[3 * k + 1], d.image.rgb[3 * k + 2]};
    }
    e.row_cos.resize(static_cast<size_t>(e.height) + 1);
    for (int j = 0; j <= e.height; ++j)
    {
        e.row_cos[static_cast<size_t>(j)] = std::cos(std::numbers::pi * j / e.height);
    }
    e.row_cos.front() = 1;
    e.row_cos.back() = -1;
    const auto luminance = [](const color& c) { return 0.2126 * c.x + 0.7152 * c.y + 0.0722 * c.z; };
    e.cell_chance.resize(n);
    double total = 0;
    for (int j = 0; j < e.height; ++j)
    {
        const double omega = 2 * std::numbers::pi / e.width * (e.row_cos[static_cast<size_t>(j)] - e.row_cos[static_cast<size_t>(j) + 1]);
        for (int i = 0; i < e.width; ++i)
        {
            const size_t c = static_cast<size_t>(j) * e.width + i;
            e.cell_chance[c] = luminance(e.texels[c]) * omega;
            total += e.cell_chance[c];
        }
    }
    e.total = total;
    e.pdf.resize(n);
    e.cell_cdf.resize(n);
    double run = 0;
    for (size_t c = 0; c < n; ++c)
    {
        e.pdf[c] = total > 0 ? luminance(e.texels[c]) / total : 0.0;
        run += e.cell_chance[c];
        e.cell_cdf[c] = run;
    }
    return e;
}
} // namespace oracle
