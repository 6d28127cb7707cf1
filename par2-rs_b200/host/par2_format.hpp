// par2_format.hpp -- the PAR2 on-disk format around the GPU codec: packet
// writing and parsing, volume naming and block counts, with the behaviour of
// par2-rs:
//
//   packet layout, bodies, File ID, set ID     writer.rs:23-264
//   File ID order (little-endian compare)      parser.rs:556-565
//   scan / parse / volume discovery / order    parser.rs:181-547, 566-800
//   volume split and file names                volumes.rs:27-210
//   block size, block and recovery counts      creator.rs:30-67, 261-352
//
// The create and repair pipelines over it are in par2_pipeline.hpp.
#pragma once
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <filesystem>
#include <map>
#include <string>
#include <vector>

#include "par2_codec.hpp"

namespace par2 {

using FileHash = std::array<uint8_t, 16>;

// ---- MD5 (RFC 1321) on the host -------------------------------------------

class Md5 {
  public:
    Md5() { reset(); }
    void reset()
    {
        s_[0] = 0x67452301u;
        s_[1] = 0xefcdab89u;
        s_[2] = 0x98badcfeu;
        s_[3] = 0x10325476u;
        n_ = 0;
        fill_ = 0;
    }
    void update(const void *data, size_t len)
    {
        const uint8_t *p = static_cast<const uint8_t *>(data);
        n_ += len;
        if (fill_) {
            const size_t take = std::min(len, size_t(64) - fill_);
            memcpy(buf_ + fill_, p, take);
            fill_ += take;
            p += take;
            len -= take;
            if (fill_ == 64) {
                block(buf_);
                fill_ = 0;
            }
        }
        for (; len >= 64; p += 64, len -= 64)
            block(p);
        if (len) {
            memcpy(buf_, p, len);
            fill_ = len;
        }
    }
    FileHash finalize()
    {
        const uint64_t bits = n_ * 8;
        const uint8_t pad = 0x80;
        update(&pad, 1);
        const uint8_t zero[64] = {};
        update(zero, fill_ <= 56 ? 56 - fill_ : 120 - fill_);
        uint8_t len[8];
        for (int i = 0; i < 8; ++i)
            len[i] = static_cast<uint8_t>(bits >> (8 * i));
        update(len, 8);
        FileHash out;
        for (int i = 0; i < 16; ++i)
            out[i] = static_cast<uint8_t>(s_[i / 4] >> (8 * (i % 4)));
        return out;
    }
    static FileHash of(const void *data, size_t len)
    {
        Md5 h;
        h.update(data, len);
        return h.finalize();
    }

  private:
    static uint32_t rotl(uint32_t x, int s) { return (x << s) | (x >> (32 - s)); }
    // one RFC 1321 block: four rounds of 16 steps, T[i] = floor(2^32 |sin(i + 1)|)
    void block(const uint8_t *p)
    {
        uint32_t x[16];
        memcpy(x, p, 64);  // little-endian host
        uint32_t a = s_[0], b = s_[1], c = s_[2], d = s_[3];
#define P2F_STEP(F, a, b, c, d, k, s, t) a = b + rotl(a + F(b, c, d) + x[k] + t, s)
#define P2F_F(b, c, d) (d ^ (b & (c ^ d)))
#define P2F_G(b, c, d) (c ^ (d & (b ^ c)))
#define P2F_H(b, c, d) (b ^ c ^ d)
#define P2F_I(b, c, d) (c ^ (b | ~d))
        P2F_STEP(P2F_F, a, b, c, d, 0, 7, 0xd76aa478);  P2F_STEP(P2F_F, d, a, b, c, 1, 12, 0xe8c7b756);
        P2F_STEP(P2F_F, c, d, a, b, 2, 17, 0x242070db); P2F_STEP(P2F_F, b, c, d, a, 3, 22, 0xc1bdceee);
        P2F_STEP(P2F_F, a, b, c, d, 4, 7, 0xf57c0faf);  P2F_STEP(P2F_F, d, a, b, c, 5, 12, 0x4787c62a);
        P2F_STEP(P2F_F, c, d, a, b, 6, 17, 0xa8304613); P2F_STEP(P2F_F, b, c, d, a, 7, 22, 0xfd469501);
        P2F_STEP(P2F_F, a, b, c, d, 8, 7, 0x698098d8);  P2F_STEP(P2F_F, d, a, b, c, 9, 12, 0x8b44f7af);
        P2F_STEP(P2F_F, c, d, a, b, 10, 17, 0xffff5bb1); P2F_STEP(P2F_F, b, c, d, a, 11, 22, 0x895cd7be);
        P2F_STEP(P2F_F, a, b, c, d, 12, 7, 0x6b901122); P2F_STEP(P2F_F, d, a, b, c, 13, 12, 0xfd987193);
        P2F_STEP(P2F_F, c, d, a, b, 14, 17, 0xa679438e); P2F_STEP(P2F_F, b, c, d, a, 15, 22, 0x49b40821);
        P2F_STEP(P2F_G, a, b, c, d, 1, 5, 0xf61e2562);  P2F_STEP(P2F_G, d, a, b, c, 6, 9, 0xc040b340);
        P2F_STEP(P2F_G, c, d, a, b, 11, 14, 0x265e5a51); P2F_STEP(P2F_G, b, c, d, a, 0, 20, 0xe9b6c7aa);
        P2F_STEP(P2F_G, a, b, c, d, 5, 5, 0xd62f105d);  P2F_STEP(P2F_G, d, a, b, c, 10, 9, 0x02441453);
        P2F_STEP(P2F_G, c, d, a, b, 15, 14, 0xd8a1e681); P2F_STEP(P2F_G, b, c, d, a, 4, 20, 0xe7d3fbc8);
        P2F_STEP(P2F_G, a, b, c, d, 9, 5, 0x21e1cde6);  P2F_STEP(P2F_G, d, a, b, c, 14, 9, 0xc33707d6);
        P2F_STEP(P2F_G, c, d, a, b, 3, 14, 0xf4d50d87); P2F_STEP(P2F_G, b, c, d, a, 8, 20, 0x455a14ed);
        P2F_STEP(P2F_G, a, b, c, d, 13, 5, 0xa9e3e905); P2F_STEP(P2F_G, d, a, b, c, 2, 9, 0xfcefa3f8);
        P2F_STEP(P2F_G, c, d, a, b, 7, 14, 0x676f02d9); P2F_STEP(P2F_G, b, c, d, a, 12, 20, 0x8d2a4c8a);
        P2F_STEP(P2F_H, a, b, c, d, 5, 4, 0xfffa3942);  P2F_STEP(P2F_H, d, a, b, c, 8, 11, 0x8771f681);
        P2F_STEP(P2F_H, c, d, a, b, 11, 16, 0x6d9d6122); P2F_STEP(P2F_H, b, c, d, a, 14, 23, 0xfde5380c);
        P2F_STEP(P2F_H, a, b, c, d, 1, 4, 0xa4beea44);  P2F_STEP(P2F_H, d, a, b, c, 4, 11, 0x4bdecfa9);
        P2F_STEP(P2F_H, c, d, a, b, 7, 16, 0xf6bb4b60); P2F_STEP(P2F_H, b, c, d, a, 10, 23, 0xbebfbc70);
        P2F_STEP(P2F_H, a, b, c, d, 13, 4, 0x289b7ec6); P2F_STEP(P2F_H, d, a, b, c, 0, 11, 0xeaa127fa);
        P2F_STEP(P2F_H, c, d, a, b, 3, 16, 0xd4ef3085); P2F_STEP(P2F_H, b, c, d, a, 6, 23, 0x04881d05);
        P2F_STEP(P2F_H, a, b, c, d, 9, 4, 0xd9d4d039);  P2F_STEP(P2F_H, d, a, b, c, 12, 11, 0xe6db99e5);
        P2F_STEP(P2F_H, c, d, a, b, 15, 16, 0x1fa27cf8); P2F_STEP(P2F_H, b, c, d, a, 2, 23, 0xc4ac5665);
        P2F_STEP(P2F_I, a, b, c, d, 0, 6, 0xf4292244);  P2F_STEP(P2F_I, d, a, b, c, 7, 10, 0x432aff97);
        P2F_STEP(P2F_I, c, d, a, b, 14, 15, 0xab9423a7); P2F_STEP(P2F_I, b, c, d, a, 5, 21, 0xfc93a039);
        P2F_STEP(P2F_I, a, b, c, d, 12, 6, 0x655b59c3); P2F_STEP(P2F_I, d, a, b, c, 3, 10, 0x8f0ccc92);
        P2F_STEP(P2F_I, c, d, a, b, 10, 15, 0xffeff47d); P2F_STEP(P2F_I, b, c, d, a, 1, 21, 0x85845dd1);
        P2F_STEP(P2F_I, a, b, c, d, 8, 6, 0x6fa87e4f);  P2F_STEP(P2F_I, d, a, b, c, 15, 10, 0xfe2ce6e0);
        P2F_STEP(P2F_I, c, d, a, b, 6, 15, 0xa3014314); P2F_STEP(P2F_I, b, c, d, a, 13, 21, 0x4e0811a1);
        P2F_STEP(P2F_I, a, b, c, d, 4, 6, 0xf7537e82);  P2F_STEP(P2F_I, d, a, b, c, 11, 10, 0xbd3af235);
        P2F_STEP(P2F_I, c, d, a, b, 2, 15, 0x2ad7d2bb); P2F_STEP(P2F_I, b, c, d, a, 9, 21, 0xeb86d391);
#undef P2F_STEP
#undef P2F_F
#undef P2F_G
#undef P2F_H
#undef P2F_I
        s_[0] += a;
        s_[1] += b;
        s_[2] += c;
        s_[3] += d;
    }
    uint32_t s_[4];
    uint64_t n_;
    uint8_t buf_[64];
    size_t fill_;
};

// ---- packets (writer.rs) ----------------------------------------------------

namespace packet_types {
inline const std::array<uint8_t, 16> MAIN = {'P', 'A', 'R', ' ', '2', '.', '0', 0,
                                             'M', 'a', 'i', 'n', 0,   0,   0,   0};
inline const std::array<uint8_t, 16> FILE_DESC = {'P', 'A', 'R', ' ', '2', '.', '0', 0,
                                                  'F', 'i', 'l', 'e', 'D', 'e', 's', 'c'};
inline const std::array<uint8_t, 16> IFSC = {'P', 'A', 'R', ' ', '2', '.', '0', 0,
                                             'I', 'F', 'S', 'C', 0,   0,   0,   0};
inline const std::array<uint8_t, 16> RECV_SLICE = {'P', 'A', 'R', ' ', '2', '.', '0', 0,
                                                   'R', 'e', 'c', 'v', 'S', 'l', 'i', 'c'};
inline const std::array<uint8_t, 16> CREATOR = {'P', 'A', 'R', ' ', '2', '.', '0', 0,
                                                'C', 'r', 'e', 'a', 't', 'o', 'r', 0};
}  // namespace packet_types

inline const uint8_t kPar2Magic[8] = {'P', 'A', 'R', '2', 0, 'P', 'K', 'T'};

// The creator text par2-rs writes (creator.rs:500-504): files written with it
// are byte-identical to the reference's.
inline const char *kReferenceCreator = "par2-rs v0.1.0 https://github.com/zephleggett/par2-rs";

struct FileInfo {
    FileHash file_id{};
    FileHash hash{};      // MD5 of the whole file
    FileHash hash_16k{};  // MD5 of the first 16 KiB
    uint64_t length = 0;
    std::string name;
};

struct SliceChecksum {
    FileHash md5{};
    uint32_t crc32 = 0;
};

inline void put_le(std::vector<uint8_t> &v, uint64_t x, int bytes)
{
    for (int i = 0; i < bytes; ++i)
        v.push_back(static_cast<uint8_t>(x >> (8 * i)));
}
inline uint64_t get_le(const uint8_t *p, int bytes)
{
    uint64_t x = 0;
    for (int i = bytes - 1; i >= 0; --i)
        x = x << 8 | p[i];
    return x;
}

// MD5(hash_16k || length LE || name) (writer.rs:55-63)
inline FileHash compute_file_id(const FileHash &hash_16k, uint64_t length, const std::string &name)
{
    Md5 h;
    h.update(hash_16k.data(), 16);
    uint8_t len[8];
    for (int i = 0; i < 8; ++i)
        len[i] = static_cast<uint8_t>(length >> (8 * i));
    h.update(len, 8);
    h.update(name.data(), name.size());
    return h.finalize();
}

inline FileHash compute_recovery_set_id(const std::vector<uint8_t> &main_body)
{
    return Md5::of(main_body.data(), main_body.size());
}

// par2cmdline's File ID order: the ID as a little-endian 128-bit number
inline bool file_id_less(const FileHash &a, const FileHash &b)
{
    for (int i = 15; i >= 0; --i)
        if (a[i] != b[i])
            return a[i] < b[i];
    return false;
}

// header (magic, length, MD5 of set id + type + body, set id, type) + body
// padded with zeros to a multiple of 4 (writer.rs:92-123)
inline void write_packet(std::vector<uint8_t> &out, const std::array<uint8_t, 16> &type,
                         const FileHash &set_id, std::vector<uint8_t> body)
{
    while (body.size() % 4)
        body.push_back(0);
    Md5 h;
    h.update(set_id.data(), 16);
    h.update(type.data(), 16);
    h.update(body.data(), body.size());
    const FileHash md5 = h.finalize();
    out.insert(out.end(), kPar2Magic, kPar2Magic + 8);
    put_le(out, 64 + body.size(), 8);
    out.insert(out.end(), md5.begin(), md5.end());
    out.insert(out.end(), set_id.begin(), set_id.end());
    out.insert(out.end(), type.begin(), type.end());
    out.insert(out.end(), body.begin(), body.end());
}

// block size u64, file count u32, File IDs in par2cmdline order (writer.rs:142-168)
inline std::vector<uint8_t> build_main_packet_body(uint64_t block_size, std::vector<FileHash> ids)
{
    std::vector<uint8_t> b;
    put_le(b, block_size, 8);
    put_le(b, ids.size(), 4);
    std::sort(ids.begin(), ids.end(), file_id_less);
    for (const FileHash &id : ids)
        b.insert(b.end(), id.begin(), id.end());
    return b;
}

// File ID, MD5, MD5 16 KiB, length, name and a NUL (writer.rs:192-221); the
// padding to 4 comes from write_packet, so a name whose length is a multiple
// of 4 is followed by four zero bytes, as par2-rs writes it.
inline std::vector<uint8_t> file_desc_body(const FileInfo &f)
{
    std::vector<uint8_t> b(f.file_id.begin(), f.file_id.end());
    b.insert(b.end(), f.hash.begin(), f.hash.end());
    b.insert(b.end(), f.hash_16k.begin(), f.hash_16k.end());
    put_le(b, f.length, 8);
    b.insert(b.end(), f.name.begin(), f.name.end());
    b.push_back(0);
    return b;
}

inline std::vector<uint8_t> ifsc_body(const FileHash &file_id, const std::vector<SliceChecksum> &cs)
{
    std::vector<uint8_t> b(file_id.begin(), file_id.end());
    for (const SliceChecksum &c : cs) {
        b.insert(b.end(), c.md5.begin(), c.md5.end());
        put_le(b, c.crc32, 4);
    }
    return b;
}

inline std::vector<uint8_t> recovery_body(uint32_t exponent, const uint8_t *data, size_t n)
{
    std::vector<uint8_t> b;
    b.reserve(4 + n);
    put_le(b, exponent, 4);
    b.insert(b.end(), data, data + n);
    return b;
}

// ---- sizes (creator.rs) -----------------------------------------------------

// ~2000 blocks, 2 KiB .. 4 MiB, a multiple of 4, at most 65535 blocks (creator.rs:30-67)
inline uint64_t calculate_block_size(uint64_t total)
{
    const uint64_t kMin = 2048, kMax = 4u << 20, kTarget = 2000, kMaxBlocks = 65535;
    if (total == 0)
        return kMin;
    uint64_t bs = total / kTarget;
    const uint64_t min_for_field = (total + kMaxBlocks - 1) / kMaxBlocks;
    if (bs % 4)
        bs = (bs / 4 + 1) * 4;
    uint64_t min_block = std::max(min_for_field, kMin);
    if (min_block % 4)
        min_block = (min_block / 4 + 1) * 4;
    if (min_block > kMax)
        bs = min_block;
    else
        bs = std::max(std::clamp(bs, kMin, kMax), min_block);
    return bs;
}

// ceil(floor(data_bytes * (double(float percent) / 100)) / block_size)
// (creator.rs:326-330: f32 percent widened to f64)
inline uint64_t recovery_block_count(uint64_t data_blocks, uint64_t block_size, float percent)
{
    const double pct = static_cast<double>(percent) / 100.0;
    const uint64_t rec_bytes = static_cast<uint64_t>(static_cast<double>(data_blocks * block_size) * pct);
    return (rec_bytes + block_size - 1) / block_size;
}

// ---- volumes (volumes.rs) ---------------------------------------------------

enum class VolumeScheme { Single, Exponential };

struct VolumeInfo {
    std::filesystem::path path;
    uint32_t exponent_start = 0, exponent_end = 0;
    std::vector<uint32_t> exponents;  // recovery slices in this file
};

inline size_t calculate_padding_width(uint32_t max_exponent)
{
    size_t w = 0;
    for (uint32_t n = max_exponent; n; n /= 10)
        ++w;
    return w ? w : 1;
}

// base.volSTART+COUNT.par2, both zero-padded to `width` (volumes.rs:65-78)
inline std::string generate_volume_filename(const std::string &base, uint32_t start, uint32_t end,
                                            size_t width)
{
    char a[32], c[32];
    snprintf(a, sizeof a, "%0*u", static_cast<int>(width), start);
    snprintf(c, sizeof c, "%0*u", static_cast<int>(width), end - start + 1);
    return base + ".vol" + a + "+" + c + ".par2";
}

// exponents: ascending recovery exponents.  Single: one file; Exponential: 1,
// 2, 4, ... slices per file, at most 1024 (volumes.rs:90-210)
inline std::vector<VolumeInfo> split_into_volumes(const std::vector<uint32_t> &exponents,
                                                  VolumeScheme scheme,
                                                  const std::filesystem::path &base_path)
{
    std::vector<VolumeInfo> vols;
    if (exponents.empty())
        return vols;
    std::string base = base_path.stem().string();
    if (base.empty())
        base = "archive";
    std::filesystem::path parent = base_path.parent_path();
    if (parent.empty())
        parent = ".";
    const uint32_t max_e = exponents.back();
    const size_t width = calculate_padding_width(max_e);
    if (scheme == VolumeScheme::Single) {
        VolumeInfo v;
        v.path = parent / generate_volume_filename(base, 0, max_e, width);
        v.exponent_start = 0;
        v.exponent_end = max_e;
        v.exponents = exponents;
        vols.push_back(v);
        return vols;
    }
    size_t target = 1;
    VolumeInfo cur;
    for (uint32_t e : exponents) {
        if (cur.exponents.empty())
            cur.exponent_start = e;
        cur.exponents.push_back(e);
        cur.exponent_end = e;
        if (cur.exponents.size() >= target) {
            cur.path = parent / generate_volume_filename(base, cur.exponent_start, cur.exponent_end, width);
            vols.push_back(cur);
            cur = VolumeInfo();
            target = std::min<size_t>(target * 2, 1024);
        }
    }
    if (!cur.exponents.empty()) {
        cur.path = parent / generate_volume_filename(base, cur.exponent_start, cur.exponent_end, width);
        vols.push_back(cur);
    }
    return vols;
}

// ---- parser (parser.rs) -----------------------------------------------------

struct RecoveryRef {
    uint32_t exponent = 0;
    std::filesystem::path file;
    uint64_t data_offset = 0, data_length = 0;
};

class Par2File {
  public:
    FileHash recovery_set_id{};
    uint64_t block_size = 0;
    std::map<FileHash, FileInfo> files;
    std::vector<FileInfo> files_in_order;   // canonical input-slice order
    std::vector<RecoveryRef> recovery_blocks;
    std::map<FileHash, std::vector<SliceChecksum>> slice_checksums;
    std::vector<FileHash> main_order;       // the Main packet's File ID list
    std::vector<std::filesystem::path> set_files;  // this file and the volumes read with it

    // Parses `path`, then every other *.par2 in its directory with the same
    // recovery set ID (parser.rs:181-547).  Packets with a bad magic, length or
    // MD5 are skipped; RecvSlic data is referenced, not read.
    static Par2File load(const std::filesystem::path &path, bool scan_volumes = true)
    {
        Par2File p;
        const uint64_t size = file_size(path);
        if (size == 0)
            throw Par2Error("Invalid PAR2 file: empty file");
        std::vector<std::pair<uint64_t, uint64_t>> deferred;
        p.scan(path, size, true, &deferred);
        if (p.recovery_set_id == FileHash{})
            throw Par2Error("Invalid PAR2 file: no main packet");
        if (p.block_size == 0)
            throw Par2Error("Invalid PAR2 file: block size missing or zero");
        if (p.block_size % 4)
            throw Par2Error("Invalid PAR2 file: block size must be multiple of 4");
        for (const auto &d : deferred)
            if (d.second >= 68)
                p.add_recovery(path, d.first);
        p.set_files.push_back(path);
        if (scan_volumes) {
            std::filesystem::path dir = path.parent_path();
            if (dir.empty())
                dir = ".";
            std::vector<std::filesystem::path> others;
            for (const auto &e : std::filesystem::directory_iterator(dir)) {
                std::string ext = e.path().extension().string();
                std::transform(ext.begin(), ext.end(), ext.begin(), ::tolower);
                if (ext == ".par2" && !std::filesystem::equivalent(e.path(), path))
                    others.push_back(e.path());
            }
            std::sort(others.begin(), others.end());
            for (const auto &v : others) {
                FileHash id{};
                if (first_set_id(v, &id) && id == p.recovery_set_id) {
                    Par2File vol;
                    vol.block_size = p.block_size;
                    vol.scan(v, file_size(v), false, nullptr);
                    p.recovery_blocks.insert(p.recovery_blocks.end(), vol.recovery_blocks.begin(),
                                             vol.recovery_blocks.end());
                    p.set_files.push_back(v);
                }
            }
        }
        p.order_files();
        return p;
    }

    std::vector<uint8_t> read_recovery(const RecoveryRef &r, uint64_t offset, uint64_t n) const
    {
        std::vector<uint8_t> out(n);
        read_recovery_into(r, offset, n, out.data());
        return out;
    }
    // The same into caller memory (safe to call from several threads).
    void read_recovery_into(const RecoveryRef &r, uint64_t offset, uint64_t n, uint8_t *out) const
    {
        FILE *f = fopen(r.file.string().c_str(), "rb");
        if (!f || fseeko(f, static_cast<off_t>(r.data_offset + offset), SEEK_SET) != 0 ||
            (n && fread(out, 1, n, f) != n)) {
            if (f)
                fclose(f);
            throw Par2Error("Failed to read recovery slice from " + r.file.string());
        }
        fclose(f);
    }

  private:
    static uint64_t file_size(const std::filesystem::path &p)
    {
        std::error_code ec;
        const auto n = std::filesystem::file_size(p, ec);
        if (ec)
            throw Par2Error("Cannot open " + p.string());
        return n;
    }
    static bool first_set_id(const std::filesystem::path &p, FileHash *id)
    {
        uint8_t h[64];
        FILE *f = fopen(p.string().c_str(), "rb");
        if (!f)
            return false;
        const bool ok = fread(h, 1, 64, f) == 64 && memcmp(h, kPar2Magic, 8) == 0;
        fclose(f);
        if (ok)
            memcpy(id->data(), h + 32, 16);
        return ok;
    }
    void add_recovery(const std::filesystem::path &path, uint64_t pos)
    {
        FILE *f = fopen(path.string().c_str(), "rb");
        uint8_t e[4];
        if (f && fseeko(f, static_cast<off_t>(pos + 64), SEEK_SET) == 0 && fread(e, 1, 4, f) == 4) {
            RecoveryRef r;
            r.exponent = static_cast<uint32_t>(get_le(e, 4));
            r.file = path;
            r.data_offset = pos + 68;
            r.data_length = block_size;
            recovery_blocks.push_back(r);
        }
        if (f)
            fclose(f);
    }
    void scan(const std::filesystem::path &path, uint64_t size, bool full,
              std::vector<std::pair<uint64_t, uint64_t>> *deferred)
    {
        FILE *f = fopen(path.string().c_str(), "rb");
        if (!f)
            throw Par2Error("Cannot open " + path.string());
        uint64_t pos = 0;
        std::vector<uint8_t> body;
        while (pos < size) {
            uint8_t h[64];
            if (fseeko(f, static_cast<off_t>(pos), SEEK_SET) != 0 || fread(h, 1, 64, f) < 64)
                break;
            if (memcmp(h, kPar2Magic, 8) != 0) {
                ++pos;
                continue;
            }
            if (full && recovery_set_id == FileHash{})
                memcpy(recovery_set_id.data(), h + 32, 16);
            const uint64_t len = get_le(h + 8, 8);
            if (len < 64 || len > size - pos) {
                ++pos;
                continue;
            }
            const uint64_t next = pos + len + (len % 4 ? 4 - len % 4 : 0);
            if (memcmp(h + 48, packet_types::RECV_SLICE.data(), 16) == 0) {
                if (block_size == 0) {
                    if (deferred)
                        deferred->push_back({pos, len});
                } else if (len >= 68) {
                    add_recovery(path, pos);
                }
                pos = next;
                continue;
            }
            if (!full) {
                pos = next;
                continue;
            }
            body.resize(len - 64);
            if (fread(body.data(), 1, body.size(), f) < body.size())
                break;
            Md5 m;
            m.update(h + 32, 32);
            m.update(body.data(), body.size());
            if (m.finalize() != *reinterpret_cast<const FileHash *>(h + 16)) {
                pos = next;  // corrupted packet
                continue;
            }
            parse_body(h + 48, body);
            pos = next;
        }
        fclose(f);
    }
    void parse_body(const uint8_t *type, const std::vector<uint8_t> &b)
    {
        if (memcmp(type, packet_types::MAIN.data(), 16) == 0 && b.size() >= 8) {
            block_size = get_le(b.data(), 8);
            if (b.size() >= 12 && main_order.empty()) {
                const uint64_t n = get_le(b.data() + 8, 4);
                for (uint64_t i = 0; i < n && 12 + 16 * (i + 1) <= b.size(); ++i) {
                    FileHash id;
                    memcpy(id.data(), b.data() + 12 + 16 * i, 16);
                    main_order.push_back(id);
                }
            }
        } else if (memcmp(type, packet_types::FILE_DESC.data(), 16) == 0 && b.size() >= 56) {
            FileInfo fi;
            memcpy(fi.file_id.data(), b.data(), 16);
            memcpy(fi.hash.data(), b.data() + 16, 16);
            memcpy(fi.hash_16k.data(), b.data() + 32, 16);
            fi.length = get_le(b.data() + 48, 8);
            size_t e = 56;
            while (e < b.size() && b[e])
                ++e;
            fi.name.assign(reinterpret_cast<const char *>(b.data() + 56), e - 56);
            if (files.emplace(fi.file_id, fi).second)
                files_in_order.push_back(fi);
        } else if (memcmp(type, packet_types::IFSC.data(), 16) == 0 && b.size() >= 16) {
            FileHash id;
            memcpy(id.data(), b.data(), 16);
            std::vector<SliceChecksum> cs;
            for (size_t o = 16; o + 20 <= b.size(); o += 20) {
                SliceChecksum c;
                memcpy(c.md5.data(), b.data() + o, 16);
                c.crc32 = static_cast<uint32_t>(get_le(b.data() + o + 16, 4));
                cs.push_back(c);
            }
            slice_checksums[id] = cs;
        }
    }
    // Main packet order first, then par2cmdline's File ID order (parser.rs:566-590)
    void order_files()
    {
        std::map<FileHash, size_t> rank;
        for (size_t i = 0; i < main_order.size(); ++i)
            rank.emplace(main_order[i], i);
        auto r = [&](const FileHash &id) {
            auto it = rank.find(id);
            return it == rank.end() ? SIZE_MAX : it->second;
        };
        std::stable_sort(files_in_order.begin(), files_in_order.end(),
                         [&](const FileInfo &a, const FileInfo &b) {
                             const size_t ra = r(a.file_id), rb = r(b.file_id);
                             return ra != rb ? ra < rb : file_id_less(a.file_id, b.file_id);
                         });
    }
};

}  // namespace par2
