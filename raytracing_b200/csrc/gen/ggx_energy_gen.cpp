// Build-time generator of the GGX energy table (run by raytracing_b200/build.py; the output is compiled into the
// library as constant data): E_ss(mu, r), the light a white GGX conductor keeps after one bounce among its facets, for
// Turquin's multiple-scattering compensation (Turquin 2019; the reference's ggx.cuh:202-236 reads a table of the same
// nodes: sqrt(mu) = i/31 columns, r = j/31 rows, row 0 and column 0 equal to 1).
//
// E = the mean over the visible normals of the sample weight G2/G1 (F = 1), integrated on the sampler's own two
// parameters (Dupuy & Benyoub's spherical caps): the azimuth by the trapezoidal rule, which is spectrally accurate for
// a periodic integrand, and for each azimuth the valid cap heights [0, u*] (the reflected light falls below the horizon
// past u*, found by bisection) by 24-point Gauss-Legendre on three sub-intervals. Double precision throughout.
#include <array>
#include <cmath>
#include <cstdio>
#include <thread>
#include <vector>

namespace
{
struct v3
{
    double x, y, z;
};
v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
v3 operator*(double t, v3 a) { return {t * a.x, t * a.y, t * a.z}; }
double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
v3 unit(v3 a) { return (1 / std::sqrt(dot(a, a))) * a; }

double smith_a(double c, double a2) { return std::sqrt(c * c * (1 - a2) + a2); }

// The weight G2/G1 of the cap sample (u1, u2) for the view v = (sin, 0, mu) about n = +z, or < 0 if absorbed
double weight(double mu, double alpha, double u1, double u2)
{
    const v3 n{0, 0, 1};
    const v3 v{std::sqrt(std::fmax(0.0, 1 - mu * mu)), 0, mu};
    const double cv = mu;
    const v3 vs = unit(alpha * (v - cv * n) + cv * n);
    const double zs = vs.z;
    const double z = (1 - u2) * (1 + zs) - zs;
    const double st = std::sqrt(std::fmax(0.0, 1 - z * z));
    const double phi = 2 * M_PI * u1;
    const v3 c{st * std::cos(phi), st * std::sin(phi), z};
    const v3 hs = c + vs;
    const double hn = hs.z;
    const v3 m{alpha * hs.x, alpha * hs.y, std::fmax(0.0, hn)};
    const double m2 = dot(m, m);
    if (!(m2 > 0))
    {
        return -1;
    }
    const v3 h = (1 / std::sqrt(m2)) * m;
    const double vh = dot(v, h);
    const v3 l = (2 * vh) * h - v;
    const double cl = l.z;
    if (!(cl > 0) || !(vh > 0))
    {
        return -1;
    }
    const double a2 = alpha * alpha;
    const double av = smith_a(cv, a2);
    const double al = smith_a(cl, a2);
    return cl * (cv + av) / (cl * av + cv * al);
}

double energy(double mu, double r)
{
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
    const double alpha = r * r;
    const int azimuths = 256;
    const int scan = 128; // heights probed per azimuth to find where the light leaves and re-enters the hemisphere
    double total = 0;
    const auto valid = [&](double u1, double u2) { return weight(mu, alpha, u1, u2) >= 0; };
    for (int a = 0; a < azimuths; ++a)
    {
        const double u1 = (a + 0.5) / azimuths;
        // The valid heights: probe, bisect every change of validity, then integrate each valid piece
        std::vector<double> edges{0.0};
        bool inside = valid(u1, 0.0);
        std::vector<std::pair<double, double>> pieces;
        double start = 0.0;
        for (int k = 1; k <= scan; ++k)
        {
            const double u = static_cast<double>(k) / scan;
            const bool now = valid(u1, u);
            if (now != inside)
            {
                double lo = static_cast<double>(k - 1) / scan, hi = u;
                for (int it = 0; it < 55; ++it)
                {
                    const double mid = 0.5 * (lo + hi);
                    (valid(u1, mid) == inside ? lo : hi) = mid;
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
        for (const auto& [p0, p1] : pieces)
        {
            // Gauss-Legendre on four equal parts of the piece
            for (int part = 0; part < 4; ++part)
            {
                const double a0 = p0 + (p1 - p0) * part / 4;
                const double b0 = p0 + (p1 - p0) * (part + 1) / 4;
                for (size_t k = 0; k < x.size(); ++k)
                {
                    const double wv = weight(mu, alpha, u1, 0.5 * (a0 + b0) + 0.5 * (b0 - a0) * x[k]);
                    total += 0.5 * (b0 - a0) * w[k] * (wv > 0 ? wv : 0.0);
                }
            }
        }
    }
    return total / azimuths;
}
} // namespace

int main(int argc, char** argv)
{
    constexpr int size = 32;
    std::vector<double> table(size * size, 1.0);
    std::vector<std::thread> workers;
    for (int j = 1; j < size; ++j)
    {
        workers.emplace_back([&table, j] {
            for (int i = 1; i < size; ++i)
            {
                const double s = static_cast<double>(i) / (size - 1);
                table[static_cast<size_t>(j * size + i)] = energy(s * s, static_cast<double>(j) / (size - 1));
            }
        });
    }
    for (std::thread& t : workers)
    {
        t.join();
    }
    FILE* f = argc > 1 ? std::fopen(argv[1], "w") : stdout;
    if (!f)
    {
        return 1;
    }
    std::fprintf(f, "// Generated by csrc/gen/ggx_energy_gen.cpp at build time: E_ss(mu, r) of a white GGX conductor,\n");
    std::fprintf(f, "// [j * 32 + i] for r = j/31 and sqrt(mu) = i/31\n#pragma once\n");
    std::fprintf(f, "#define RTB_GGX_ENERGY_TABLE \\\n");
    for (int k = 0; k < size * size; ++k)
    {
        std::fprintf(f, "%.9ef%s", table[static_cast<size_t>(k)], k + 1 < size * size ? ", " : "");
        if (k % 8 == 7 && k + 1 < size * size)
        {
            std::fprintf(f, "\\\n");
        }
    }
    std::fprintf(f, "\n");
    if (f != stdout)
    {
        std::fclose(f);
    }
    return 0;
}
