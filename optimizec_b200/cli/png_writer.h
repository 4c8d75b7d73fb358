// png_writer.h — RGB8 PNG encoder of the mem_cuda CLI's movie frames (no compression library).
#pragma once

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

// PNG (ISO/IEC 15948) RGB8 image: filter byte 0 per row, zlib stream (RFC 1950) of stored deflate
// blocks (RFC 1951 BTYPE 00), one IDAT chunk. CRC-32 is the reflected 0xEDB88320 polynomial,
// table-driven; Adler-32 defers the modulo over runs of 5552 bytes, the longest run for which
// the 32-bit sums cannot overflow.
class PngWriter {
  public:
    PngWriter()
    {
        for (uint32_t n = 0; n < 256; ++n) {
            uint32_t c = n;
            for (int k = 0; k < 8; ++k) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
            crc_table_[n] = c;
        }
    }

    bool write(const std::string &path, int w, int h, const unsigned char *rgb) const
    {
        const size_t row = (size_t)w * 3 + 1, raw = row * (size_t)h;
        const size_t nblk = std::max<size_t>(1, (raw + 65534) / 65535);
        std::vector<unsigned char> z;
        z.reserve(2 + raw + 5 * nblk + 4);
        z.push_back(0x78);  // CM 8 (deflate), 32 KB window
        z.push_back(0x01);  // no preset dictionary, FCHECK so that 0x7801 % 31 == 0
        uint32_t a = 1, b = 0;
        size_t done = 0, y = 0, x = 0;  // x: byte within the current row (0 = filter byte)
        for (size_t k = 0; k < nblk; ++k) {
            const size_t n = std::min<size_t>(65535, raw - done);
            z.push_back(k + 1 == nblk ? 1 : 0);
            z.push_back((unsigned char)(n & 255));
            z.push_back((unsigned char)(n >> 8));
            z.push_back((unsigned char)(~n & 255));
            z.push_back((unsigned char)((~n >> 8) & 255));
            for (size_t left = n; left > 0;) {
                if (x == 0) {  // filter type 0 (None) opens each row
                    z.push_back(0);
                    b = (b + a) % 65521u;  // adler of a zero byte: a unchanged
                    --left;
                    x = 1;
                    continue;
                }
                const size_t take = std::min(left, row - x);
                const unsigned char *src = rgb + y * (size_t)w * 3 + (x - 1);
                z.insert(z.end(), src, src + take);
                adler(src, take, a, b);
                left -= take;
                x += take;
                if (x == row) {
                    x = 0;
                    ++y;
                }
            }
            done += n;
        }
        put32(z, (b << 16) | a);

        FILE *fp = std::fopen(path.c_str(), "wb");
        if (!fp) {
            std::fprintf(stderr, "PNG %s: %s\n", path.c_str(), std::strerror(errno));
            return false;
        }
        static const unsigned char sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
        std::vector<unsigned char> ihdr;
        put32(ihdr, (uint32_t)w);
        put32(ihdr, (uint32_t)h);
        ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // depth 8, truecolour, deflate, filter 0, no interlace
        bool ok = std::fwrite(sig, 1, 8, fp) == 8 && chunk(fp, "IHDR", ihdr) && chunk(fp, "IDAT", z) &&
                  chunk(fp, "IEND", {});
        ok = (std::fclose(fp) == 0) && ok;
        if (!ok) std::fprintf(stderr, "PNG %s: write failed\n", path.c_str());
        return ok;
    }

  private:
    uint32_t crc_table_[256];

    static void put32(std::vector<unsigned char> &v, uint32_t x)
    {
        for (int s = 24; s >= 0; s -= 8) v.push_back((unsigned char)(x >> s));
    }

    // a and b enter and leave reduced mod 65521
    static void adler(const unsigned char *p, size_t n, uint32_t &a, uint32_t &b)
    {
        while (n > 0) {
            const size_t run = std::min<size_t>(n, 5552);
            for (size_t i = 0; i < run; ++i) {
                a += p[i];
                b += a;
            }
            a %= 65521u;
            b %= 65521u;
            p += run;
            n -= run;
        }
    }

    uint32_t crc(uint32_t c, const unsigned char *p, size_t n) const
    {
        for (size_t i = 0; i < n; ++i) c = crc_table_[(c ^ p[i]) & 255u] ^ (c >> 8);
        return c;
    }

    bool chunk(FILE *fp, const char type[5], const std::vector<unsigned char> &data) const
    {
        std::vector<unsigned char> head;
        put32(head, (uint32_t)data.size());
        head.insert(head.end(), type, type + 4);
        uint32_t c = crc(0xFFFFFFFFu, head.data() + 4, 4);
        c = crc(c, data.data(), data.size()) ^ 0xFFFFFFFFu;
        std::vector<unsigned char> tail;
        put32(tail, c);
        return std::fwrite(head.data(), 1, 8, fp) == 8 &&
               (data.empty() || std::fwrite(data.data(), 1, data.size(), fp) == data.size()) &&
               std::fwrite(tail.data(), 1, 4, fp) == 4;
    }
};
