// The display transform: an image's FP64 per-pixel sums turned into the 4 bytes per pixel a screen or a PNG shows
// (the reference's session::display, src/gpu/renderer.h:623-635 and renderer.cu:1388-1470; its kernels rgba8_kernel,
// display.cu:26, and tone_map_kernel, tonemap.cu:25, with the curves of tone_curves.cuh).
//
// This translation unit is compiled with -fmad=false (raytracing_b200/build.py), as the reference compiles its display
// units (CMakeLists.txt:159-165): no product is fused with the sum that follows it, so every operation rounds on its
// own in the order the expressions are written, and the bytes equal the reference's bit for bit. That equality is the
// specification, so the arithmetic below keeps the reference's operations, constants and evaluation order; the
// published constants are the sRGB OETF's (IEC 61966-2-1), AgX's log range, curve and matrices (Troy Sobotka's AgX;
// Benjamin Wrensch's Minimal AgX; linlin's closed form of the curve), Khronos PBR Neutral's F90, K_s, K_d and Jorge
// Jimenez's interleaved gradient noise.
//
// One thread per pixel, grid-stride: a pixel reads its 24 bytes of sums and writes one 4-byte word, so the kernel is
// bound by HBM bandwidth (28 bytes a pixel) and takes a few microseconds per megapixel.
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "host.h"

namespace rtb
{
namespace
{
// ---- the books' bytes (image.ixx to_byte; display.cu) ----------------------------------------------------------
// gamma 2 (the square root; 0 for anything not above 0, NaN included), clamped to [0, 0.999], times 256, truncated.
// Double throughout: sqrt is correctly rounded and 256·g is exact, so the byte equals the CPU writer's.
__device__ __forceinline__ uint8_t books_byte(double linear)
{
    double g = 0.0;
    if (linear > 0)
    {
        g = sqrt(linear);
    }
    if (g < 0.0)
    {
        g = 0.0;
    }
    if (g > 0.999)
    {
        g = 0.999;
    }
    return static_cast<uint8_t>(256 * g);
}

// ---- the tone maps beyond the books (float; tone_curves.cuh) ---------------------------------------------------
struct light3
{
    float r, g, b;
};

__device__ __forceinline__ float unit(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// What a curve may take: NaN, negatives and -inf to 0, +inf to a large finite number
__device__ __forceinline__ float finite_light(float v) { return v > 0.0f ? fminf(v, 3.0e38f) : 0.0f; }

// The sRGB OETF of a linear value in [0, 1]: 12.92·v below 0.0031308, else 1.055·v^(1/2.4) − 0.055; 1 gives 1
__device__ __forceinline__ float srgb_oetf(float v)
{
    if (v >= 1.0f)
    {
        return 1.0f;
    }
    if (v <= 0.0031308f)
    {
        return 12.92f * v;
    }
    return 1.055f * powf(v, 1.0f / 2.4f) - 0.055f;
}

// AgX: a linear value's place on the 16.5-stop log2 scale around middle grey, in [0, 1]
__device__ __forceinline__ float agx_scale_position(float v)
{
    constexpr float lowest_ev = -12.47393f;
    constexpr float highest_ev = 4.026069f;
    return unit((log2f(v) - lowest_ev) / (highest_ev - lowest_ev));
}

// AgX's S-curve in closed form: 0.5 + 2d·(1 + a·|d|^b)^c with d = x − 10/16.5, (a, b, c) = (59.507875, 3, −1/3) below
// the middle and (69.86278913545539, 13/4, −4/13) above; |d|^(13/4) as |d|³·√√|d|
__device__ __forceinline__ float agx_s_curve(float x)
{
    constexpr float middle = 0.6060606060606061f;
    const float d = x - middle;
    const float m = fabsf(d);
    const float m3 = m * m * m;
    if (x <= middle)
    {
        return 0.5f + 2.0f * d * rcbrtf(1.0f + 59.507875f * m3);
    }
    return 0.5f + 2.0f * d * powf(1.0f + 69.86278913545539f * (m3 * sqrtf(sqrtf(m))), -4.0f / 13.0f);
}

// AgX of a color: the inset matrix (rows acting on the column (r, g, b)), the log scale, the curve per channel, the
// outset (the inset's inverse), each channel clamped to [0, 1]; display-encoded already
__device__ __forceinline__ light3 agx_encode(light3 c)
{
    const float ir = 0.842479062253094f * c.r + 0.0784335999999992f * c.g + 0.0792237451477643f * c.b;
    const float ig = 0.0423282422610123f * c.r + 0.878468636469772f * c.g + 0.0791661274605434f * c.b;
    const float ib = 0.0423756549057051f * c.r + 0.0784336f * c.g + 0.879142973793104f * c.b;
    const float sr = agx_s_curve(agx_scale_position(ir));
    const float sg = agx_s_curve(agx_scale_position(ig));
    const float sb = agx_s_curve(agx_scale_position(ib));
    light3 out;
    out.r = unit(1.19687900512017f * sr - 0.0980208811401368f * sg - 0.0990297440797205f * sb);
    out.g = unit(-0.0528968517574562f * sr + 1.15190312990417f * sg - 0.0989611768448433f * sb);
    out.b = unit(-0.0529716355144438f * sr - 0.0980434501171241f * sg + 1.15107367264116f * sb);
    return out;
}

// Khronos PBR Neutral (F90 = 0.04, K_s = 0.76, K_d = 0.15): the toe that takes a specular 0.04 off, then the
// brightest channel compressed above K_s, one scale and one shift for the three channels
__device__ __forceinline__ light3 neutral_encode(light3 c)
{
    constexpr float f90 = 0.04f;
    constexpr float ks = 0.8f - f90;
    constexpr float kd = 0.15f;
    const float lowest = fminf(c.r, fminf(c.g, c.b));
    const float toe = lowest <= 2.0f * f90 ? lowest - 6.25f * lowest * lowest : f90;
    light3 s{c.r - toe, c.g - toe, c.b - toe};
    const float peak = fmaxf(s.r, fmaxf(s.g, s.b));
    if (peak <= ks)
    {
        return s;
    }
    const float compressed = 1.0f - (1.0f - ks) * (1.0f - ks) / (peak + 1.0f - 2.0f * ks);
    const float fade = 1.0f / (kd * (peak - compressed) + 1.0f);
    const float scale = compressed / peak * fade;
    const float white = compressed * (1.0f - fade);
    return {s.r * scale + white, s.g * scale + white, s.b * scale + white};
}

__device__ __forceinline__ light3 tone_encode(light3 linear, int op)
{
    const light3 c{finite_light(linear.r), finite_light(linear.g), finite_light(linear.b)};
    if (op == RT_TONE_AGX)
    {
        return agx_encode(c);
    }
    if (op == RT_TONE_NEUTRAL)
    {
        const light3 n = neutral_encode(c);
        return {srgb_oetf(unit(n.r)), srgb_oetf(unit(n.g)), srgb_oetf(unit(n.b))};
    }
    return {srgb_oetf(unit(c.r)), srgb_oetf(unit(c.g)), srgb_oetf(unit(c.b))}; // RT_TONE_NONE
}

__device__ __forceinline__ float fractional(float v) { return v - floorf(v); }

// Interleaved gradient noise at pixel (x, y): the dither depends on the pixel's place alone
__device__ __forceinline__ float gradient_noise(int x, int y)
{
    return fractional(52.9829189f *
                      fractional(0.06711056f * static_cast<float>(x) + 0.00583715f * static_cast<float>(y)));
}

// round(255·v + dither) clamped to a byte; 0 and 1 are never dithered, NaN gives 0
__device__ __forceinline__ uint8_t dithered_byte(float encoded, float dither)
{
    if (!(encoded > 0.0f))
    {
        return 0;
    }
    if (encoded >= 1.0f)
    {
        return 255;
    }
    return static_cast<uint8_t>(fminf(fmaxf(floorf(255.0f * encoded + 0.5f + dither), 0.0f), 255.0f));
}

__global__ void __launch_bounds__(256) display_kernel(const double* __restrict__ sums, int64_t pixels, int width,
                                                      double scale, int op, float exposure_scale,
                                                      uchar4* __restrict__ rgba)
{
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < pixels; p += stride)
    {
        const double* s = sums + 3 * p;
        const double r = __ldcs(s);
        const double g = __ldcs(s + 1);
        const double b = __ldcs(s + 2);
        uchar4 out;
        if (op == RT_TONE_BOOKS)
        {
            out = make_uchar4(books_byte(r * scale), books_byte(g * scale), books_byte(b * scale), 255);
        }
        else
        {
            // The light of a complete pass as a PFM holds it (the sum times 1/passes in double, rounded to float),
            // then the exposure: one float multiplication, by exactly 1 at 0 EV
            const light3 light{static_cast<float>(r * scale) * exposure_scale,
                               static_cast<float>(g * scale) * exposure_scale,
                               static_cast<float>(b * scale) * exposure_scale};
            const light3 e = tone_encode(light, op);
            const int x = static_cast<int>(p % width);
            const int y = static_cast<int>(p / width);
            const float dither = gradient_noise(x, y) - 0.5f;
            out = make_uchar4(dithered_byte(e.r, dither), dithered_byte(e.g, dither), dithered_byte(e.b, dither), 255);
        }
        __stcs(rgba + p, out);
    }
}
} // namespace

void check_display(const rt_display_options& options)
{
    if (options.tone_map < RT_TONE_BOOKS || options.tone_map > RT_TONE_NEUTRAL)
    {
        fail(RT_ERR_INVALID, "tone_map must be RT_TONE_BOOKS, RT_TONE_NONE, RT_TONE_AGX or RT_TONE_NEUTRAL");
    }
    if (!(std::isfinite(options.exposure) && std::fabs(options.exposure) <= max_exposure_stops))
    {
        fail(RT_ERR_INVALID, "an exposure is a finite number of stops from -24 to 24");
    }
    if (options.tone_map == RT_TONE_BOOKS && options.exposure != 0)
    {
        fail(RT_ERR_INVALID, "the books' bytes take no exposure: it needs another tone map");
    }
}

void launch_display(const double* sums, int width, int height, double scale, const rt_display_options& options,
                    uint8_t* rgba, cudaStream_t stream)
{
    check_display(options);
    const int64_t pixels = static_cast<int64_t>(width) * height;
    if (pixels <= 0)
    {
        return;
    }
    if ((reinterpret_cast<uintptr_t>(rgba) & 3) != 0 || (reinterpret_cast<uintptr_t>(sums) & 7) != 0)
    {
        fail(RT_ERR_INVALID, "the display's bytes must be 4-byte aligned and the sums 8-byte aligned");
    }
    // 2^EV in double, rounded once to float: a whole number of stops is an exact power of two
    const auto exposure_scale = static_cast<float>(std::exp2(options.exposure));
    int device = 0, sms = 0;
    check(cudaGetDevice(&device), "querying the device");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "querying the device");
    const int64_t blocks = std::min<int64_t>((pixels + 255) / 256, static_cast<int64_t>(sms) * 8);
    display_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(sums, pixels, width, scale, options.tone_map,
                                                                      exposure_scale, reinterpret_cast<uchar4*>(rgba));
    check(cudaGetLastError(), "launching the display transform");
}
} // namespace rtb
