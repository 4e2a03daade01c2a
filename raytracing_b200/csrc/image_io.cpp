// The image files of a render and its mean radiance (the reference's image class, src/image.ixx:93-203): PFM keeps
// the linear values (ImageCompare's input), PNG the display transform's bytes, and the mean radiance is the number
// the reference's programs print after every render.
//
// The PNG is written here without a compression library: its image data is a zlib stream of stored (uncompressed)
// deflate blocks (RFC 1950/1951), each row behind filter byte 0, with the chunk CRC-32 (ISO 3309, as PNG specifies)
// and the stream's Adler-32. A decoder reads the same pixels as from the reference's stb-compressed file; the file is
// larger (3 bytes a pixel plus a few per 64 KiB), which a writer of renders can afford.
#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "host.h"

namespace rtb
{
namespace
{
enum class file_format
{
    pfm,
    png,
    unknown
};

// image.ixx format_of: by the extension, in any letter case
file_format format_of(const std::string& path)
{
    const size_t dot = path.find_last_of('.');
    const size_t slash = path.find_last_of("/\\");
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash))
    {
        return file_format::unknown;
    }
    std::string ext = path.substr(dot + 1);
    std::transform(ext.begin(), ext.end(), ext.begin(), [](unsigned char c) { return std::tolower(c); });
    return ext == "pfm" ? file_format::pfm : ext == "png" ? file_format::png : file_format::unknown;
}

class file_writer
{
public:
    explicit file_writer(const char* path) : f_(std::fopen(path, "wb"))
    {
        if (!f_)
        {
            fail(RT_ERR_RUNTIME, std::string("could not open the file ") + path);
        }
    }
    ~file_writer()
    {
        if (f_)
        {
            std::fclose(f_);
        }
    }
    void write(const void* data, size_t n)
    {
        if (n > 0 && std::fwrite(data, 1, n, f_) != n)
        {
            fail(RT_ERR_RUNTIME, "could not write the file");
        }
    }
    void close()
    {
        const int r = std::fclose(f_);
        f_ = nullptr;
        if (r != 0)
        {
            fail(RT_ERR_RUNTIME, "could not write the file");
        }
    }

private:
    std::FILE* f_;
};

// ---- PFM (image.ixx:147-168) ------------------------------------------------------------------------------------
void save_pfm(const char* path, const double* pixels, int width, int height)
{
    file_writer f(path);
    char header[64];
    const int n = std::snprintf(header, sizeof(header), "PF\n%d %d\n-1.0\n", width, height);
    f.write(header, static_cast<size_t>(n));
    std::vector<float> row(static_cast<size_t>(width) * 3);
    for (int y = height - 1; y >= 0; --y) // rows from the bottom
    {
        const double* src = pixels + static_cast<size_t>(y) * width * 3;
        for (size_t i = 0; i < row.size(); ++i)
        {
            row[i] = static_cast<float>(src[i]); // little-endian on every host this library builds for
        }
        f.write(row.data(), row.size() * sizeof(float));
    }
    f.close();
}

// ---- PNG ----------------------------------------------------------------------------------------------------------
const std::array<uint32_t, 256>& crc_table()
{
    static const std::array<uint32_t, 256> table = [] {
        std::array<uint32_t, 256> t{};
        for (uint32_t n = 0; n < 256; ++n)
        {
            uint32_t c = n;
            for (int k = 0; k < 8; ++k)
            {
                c = (c & 1) ? 0xedb88320u ^ (c >> 1) : c >> 1;
            }
            t[n] = c;
        }
        return t;
    }();
    return table;
}

uint32_t crc_update(uint32_t crc, const uint8_t* data, size_t n)
{
    const auto& t = crc_table();
    for (size_t i = 0; i < n; ++i)
    {
        crc = t[(crc ^ data[i]) & 0xff] ^ (crc >> 8);
    }
    return crc;
}

void put_be32(std::vector<uint8_t>& out, uint32_t v)
{
    out.push_back(static_cast<uint8_t>(v >> 24));
    out.push_back(static_cast<uint8_t>(v >> 16));
    out.push_back(static_cast<uint8_t>(v >> 8));
    out.push_back(static_cast<uint8_t>(v));
}

void write_chunk(file_writer& f, const char type[4], const std::vector<uint8_t>& data)
{
    std::vector<uint8_t> head;
    put_be32(head, static_cast<uint32_t>(data.size()));
    head.insert(head.end(), type, type + 4);
    f.write(head.data(), head.size());
    f.write(data.data(), data.size());
    uint32_t crc = crc_update(0xffffffffu, reinterpret_cast<const uint8_t*>(type), 4);
    crc = crc_update(crc, data.data(), data.size()) ^ 0xffffffffu;
    std::vector<uint8_t> tail;
    put_be32(tail, crc);
    f.write(tail.data(), tail.size());
}

// rgb: height rows of width * 3 bytes, from the top
void write_png(const char* path, const std::vector<uint8_t>& rgb, int width, int height)
{
    // The raw image: each row behind filter byte 0 (None)
    const size_t row_bytes = static_cast<size_t>(width) * 3;
    std::vector<uint8_t> raw;
    raw.reserve((row_bytes + 1) * static_cast<size_t>(height));
    for (int y = 0; y < height; ++y)
    {
        raw.push_back(0);
        raw.insert(raw.end(), rgb.begin() + static_cast<std::ptrdiff_t>(row_bytes * y),
                   rgb.begin() + static_cast<std::ptrdiff_t>(row_bytes * (y + 1)));
    }
    // zlib: CMF 0x78 (deflate, 32 KiB window), FLG 0x01 (check bits: 0x7801 % 31 == 0), stored blocks, Adler-32
    std::vector<uint8_t> z{0x78, 0x01};
    constexpr size_t block = 65535;
    size_t at = 0;
    do
    {
        const size_t n = std::min(block, raw.size() - at);
        const bool last = at + n == raw.size();
        z.push_back(last ? 1 : 0); // BFINAL, BTYPE 00
        z.push_back(static_cast<uint8_t>(n));
        z.push_back(static_cast<uint8_t>(n >> 8));
        z.push_back(static_cast<uint8_t>(~n));
        z.push_back(static_cast<uint8_t>(~n >> 8));
        z.insert(z.end(), raw.begin() + static_cast<std::ptrdiff_t>(at), raw.begin() + static_cast<std::ptrdiff_t>(at + n));
        at += n;
    } while (at < raw.size());
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw)
    {
        a = (a + c) % 65521u;
        b = (b + a) % 65521u;
    }
    put_be32(z, (b << 16) | a);

    file_writer f(path);
    const uint8_t signature[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    f.write(signature, sizeof(signature));
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, static_cast<uint32_t>(width));
    put_be32(ihdr, static_cast<uint32_t>(height));
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0}); // 8 bits, truecolour RGB, deflate, adaptive filtering, no interlace
    write_chunk(f, "IHDR", ihdr);
    write_chunk(f, "IDAT", z);
    write_chunk(f, "IEND", {});
    f.close();
}

// image.ixx to_byte: gamma 2, clamped to [0, 0.999], times 256 truncated (the books' bytes; display.cu's twin)
uint8_t books_byte(double linear)
{
    double g = linear > 0 ? std::sqrt(linear) : 0.0;
    g = g < 0.0 ? 0.0 : (0.999 < g ? 0.999 : g);
    return static_cast<uint8_t>(256 * g);
}

void check_size(int width, int height)
{
    if (width < 1 || height < 1 || width > 65535 * 8 || height > 65535 * 8)
    {
        fail(RT_ERR_INVALID, "an image is 1 to 524280 pixels wide and high");
    }
}
} // namespace

void save_png_rgba(const char* path, const uint8_t* rgba, int width, int height)
{
    check_size(width, height);
    const size_t n = static_cast<size_t>(width) * static_cast<size_t>(height);
    std::vector<uint8_t> rgb(n * 3);
    for (size_t i = 0; i < n; ++i)
    {
        rgb[3 * i] = rgba[4 * i];
        rgb[3 * i + 1] = rgba[4 * i + 1];
        rgb[3 * i + 2] = rgba[4 * i + 2];
    }
    write_png(path, rgb, width, height);
}

void save_image(const char* path, const double* pixels, int width, int height, const rt_display_options& options)
{
    check_size(width, height);
    check_display(options);
    const file_format format = format_of(path);
    if (format == file_format::unknown)
    {
        fail(RT_ERR_INVALID, "unknown image format: the file name must end in .png or .pfm");
    }
    if (format == file_format::pfm)
    {
        save_pfm(path, pixels, width, height);
        return;
    }
    const size_t n = static_cast<size_t>(width) * static_cast<size_t>(height);
    if (options.tone_map == RT_TONE_BOOKS)
    {
        std::vector<uint8_t> rgb(n * 3);
        for (size_t i = 0; i < n * 3; ++i)
        {
            rgb[i] = books_byte(pixels[i]);
        }
        write_png(path, rgb, width, height);
        return;
    }
    // A tone map's bytes come from the GPU's kernel (the reference computes them on the GPU only: the host's and the
    // device's powf and log2f may round differently); the pixels are already the sums times 1 / passes, so scale 1
    cudaStream_t stream = nullptr;
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "creating a CUDA stream");
    device_array<double> sums;
    device_array<uint8_t> rgba;
    std::vector<uint8_t> host(n * 4);
    try
    {
        sums.allocate_async(n * 3, stream);
        rgba.allocate_async(n * 4, stream);
        check(cudaMemcpyAsync(sums.data(), pixels, n * 3 * sizeof(double), cudaMemcpyHostToDevice, stream),
              "copying the image");
        launch_display(sums.data(), width, height, 1.0, options, rgba.data(), stream);
        check(cudaMemcpyAsync(host.data(), rgba.data(), n * 4, cudaMemcpyDeviceToHost, stream),
              "copying the display's bytes");
        check(cudaStreamSynchronize(stream), "converting the image for the display");
    }
    catch (...)
    {
        sums.release();
        rgba.release();
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
        throw;
    }
    sums.release();
    rgba.release();
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
    save_png_rgba(path, host.data(), width, height);
}

double mean_radiance(const double* pixels, int64_t pixel_count)
{
    if (pixel_count <= 0)
    {
        fail(RT_ERR_INVALID, "an image has at least one pixel");
    }
    // image.ixx average(): the colors folded in pixel order, times 1 / count; then the channels' mean
    double r = 0, g = 0, b = 0;
    for (int64_t i = 0; i < pixel_count; ++i)
    {
        r = r + pixels[3 * i];
        g = g + pixels[3 * i + 1];
        b = b + pixels[3 * i + 2];
    }
    const double inverse = 1 / static_cast<double>(pixel_count);
    return (inverse * r + inverse * g + inverse * b) / 3;
}
} // namespace rtb
