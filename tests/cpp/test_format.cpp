// Drives par2-rs_b200/host/par2_format.hpp and par2_pipeline.hpp for tests/test_format_cpp.py:
//
//   test_format parse <file.par2>             parsed set as JSON (host only)
//   test_format headers <dir> <block> <files...>
//                                             Main + FileDesc packet headers (host only)
//   test_format create <out.par2> <block> <percent> <scheme> <files...>
//                                             writes a set (GPU: IFSC + recovery)
//   test_format repair <file.par2> <dir>      verifies every slice on the GPU and
//                                             rebuilds damaged files in place
//   test_format blocksize <bytes...>          calculate_block_size of each total,
//                                             one per line (host only)
//   test_format volumes <single|exp> <n> <base>
//                                             split_into_volumes of exponents 0..n-1:
//                                             "start end count path" per volume
//   test_format volname <base> <start> <end> <width>
//                                             generate_volume_filename
//   test_format padwidth <max...>             calculate_padding_width of each
//   test_format idless <hexA> <hexB>          file_id_less(A, B) as 1 / 0
//   test_format reccount <blocks> <bs> <pct>  recovery_block_count
#include <stdio.h>

#include <set>
#include <string>

#include "../../par2-rs_b200/host/par2_pipeline.hpp"

using namespace par2;
namespace fs = std::filesystem;

static std::string hex(const uint8_t *p, size_t n)
{
    static const char *d = "0123456789abcdef";
    std::string s;
    for (size_t i = 0; i < n; ++i) {
        s += d[p[i] >> 4];
        s += d[p[i] & 15];
    }
    return s;
}
static std::string hex(const FileHash &h) { return hex(h.data(), 16); }

static int cmd_parse(const char *path)
{
    Par2File p = Par2File::load(path);
    printf("{\"set_id\": \"%s\", \"block_size\": %llu, \"files\": [", hex(p.recovery_set_id).c_str(),
           static_cast<unsigned long long>(p.block_size));
    for (size_t i = 0; i < p.files_in_order.size(); ++i) {
        const FileInfo &f = p.files_in_order[i];
        printf("%s{\"file_id\": \"%s\", \"name\": \"%s\", \"length\": %llu, \"md5\": \"%s\", "
               "\"md5_16k\": \"%s\", \"ifsc\": [",
               i ? ", " : "", hex(f.file_id).c_str(), f.name.c_str(),
               static_cast<unsigned long long>(f.length), hex(f.hash).c_str(), hex(f.hash_16k).c_str());
        const auto &cs = p.slice_checksums[f.file_id];
        for (size_t j = 0; j < cs.size(); ++j)
            printf("%s[\"%s\", %u]", j ? ", " : "", hex(cs[j].md5).c_str(), cs[j].crc32);
        printf("]}");
    }
    printf("], \"recovery\": [");
    for (size_t i = 0; i < p.recovery_blocks.size(); ++i) {
        const RecoveryRef &r = p.recovery_blocks[i];
        printf("%s[%u, \"%s\"]", i ? ", " : "", r.exponent,
               hex(Md5::of(p.read_recovery(r, 0, r.data_length).data(), r.data_length)).c_str());
    }
    printf("]}\n");
    return 0;
}

static int cmd_headers(const char *dir, uint64_t bs, int n, char **names)
{
    std::vector<FileInfo> infos;
    for (int i = 0; i < n; ++i) {
        FILE *f = fopen((fs::path(dir) / names[i]).string().c_str(), "rb");
        std::vector<uint8_t> d(fs::file_size(fs::path(dir) / names[i]));
        if (!f || (d.size() && fread(d.data(), 1, d.size(), f) != d.size()))
            return 2;
        fclose(f);
        FileInfo fi;
        fi.name = names[i];
        fi.length = d.size();
        fi.hash = Md5::of(d.data(), d.size());
        fi.hash_16k = Md5::of(d.data(), std::min<size_t>(d.size(), 16384));
        fi.file_id = compute_file_id(fi.hash_16k, fi.length, fi.name);
        infos.push_back(fi);
    }
    std::vector<FileHash> ids;
    for (const FileInfo &f : infos)
        ids.push_back(f.file_id);
    const std::vector<uint8_t> main = build_main_packet_body(bs, ids);
    const FileHash set_id = compute_recovery_set_id(main);
    std::vector<uint8_t> out;
    write_packet(out, packet_types::MAIN, set_id, main);
    printf("%s\n", hex(out.data(), 64).c_str());
    for (const FileInfo &f : infos) {
        out.clear();
        write_packet(out, packet_types::FILE_DESC, set_id, file_desc_body(f));
        printf("%s\n", hex(out.data(), 64).c_str());
    }
    return 0;
}

static int cmd_create(const char *out, uint64_t bs, float pct, const char *scheme, int n, char **files)
{
    std::vector<fs::path> in(files, files + n);
    Par2Creator c(in);
    c.with_output_path(out).with_redundancy(pct).with_volume_scheme(
        std::string(scheme) == "single" ? VolumeScheme::Single : VolumeScheme::Exponential);
    if (bs)
        c.with_block_size(bs);
    for (const fs::path &p : c.create())
        printf("%s\n", p.string().c_str());
    return 0;
}

// Verification and repair of a parsed set: the slices of every file are
// checked against the IFSC entries on the GPU (missing files count as all
// damaged), the damaged slices are rebuilt from the m lowest recovery
// exponents (repair.rs:537-604) and the files rewritten.
static int cmd_repair(const char *par2, const char *dir)
{
    Par2File p = Par2File::load(par2);
    const uint64_t bs = p.block_size;
    size_t k = 0;
    for (const FileInfo &f : p.files_in_order)
        k += static_cast<size_t>((f.length + bs - 1) / bs);
    std::vector<uint8_t> slices(k * bs, 0);
    std::vector<size_t> damaged;
    size_t g0 = 0;
    for (const FileInfo &f : p.files_in_order) {
        const size_t nb = static_cast<size_t>((f.length + bs - 1) / bs);
        const fs::path fp = fs::path(dir) / f.name;
        bool present = fs::exists(fp);
        if (present) {
            FILE *fh = fopen(fp.string().c_str(), "rb");
            const size_t want = std::min<uint64_t>(f.length, fs::file_size(fp));
            if (!fh || (want && fread(slices.data() + g0 * bs, 1, want, fh) != want))
                present = false;
            if (fh)
                fclose(fh);
        }
        const auto &cs = p.slice_checksums[f.file_id];
        std::vector<uint8_t> md5(nb * 16), ok(nb, 0);
        std::vector<uint32_t> crc(nb);
        for (size_t b = 0; b < nb && b < cs.size(); ++b) {
            memcpy(md5.data() + b * 16, cs[b].md5.data(), 16);
            crc[b] = cs[b].crc32;
        }
        if (present && nb) {
            std::vector<const uint8_t *> sp(nb);
            for (size_t b = 0; b < nb; ++b)
                sp[b] = slices.data() + (g0 + b) * bs;
            check(p2g_verify_slices(codec_ctx(), sp.data(), nb, bs, md5.data(), crc.data(), ok.data(), 0));
        }
        for (size_t b = 0; b < nb; ++b)
            if (!ok[b])
                damaged.push_back(g0 + b);
        g0 += nb;
    }
    printf("damaged %zu\n", damaged.size());
    if (damaged.empty())
        return 0;
    std::vector<RecoveryRef> recs = p.recovery_blocks;
    std::sort(recs.begin(), recs.end(),
              [](const RecoveryRef &a, const RecoveryRef &b) { return a.exponent < b.exponent; });
    if (recs.size() < damaged.size()) {
        printf("insufficient recovery: need %zu, have %zu\n", damaged.size(), recs.size());
        return 3;
    }
    Par2ReedSolomon rs(k, recs.size());
    std::vector<size_t> present, prec;
    std::vector<uint32_t> exps;
    std::set<size_t> dset(damaged.begin(), damaged.end());
    for (size_t i = 0; i < k; ++i)
        if (!dset.count(i))
            present.push_back(i);
    for (size_t q = 0; q < damaged.size(); ++q) {
        prec.push_back(k + q);
        exps.push_back(recs[q].exponent);
    }
    // exponent table indexed by recovery block number (k + q)
    ReconstructionTransform t = rs.compute_reconstruction_transform(damaged, present, prec, exps);
    rs.reconstruct_streaming_chunk(
        damaged, present, prec, t, 0, bs,
        [&](size_t idx, size_t off, size_t n) {
            if (idx < k)
                return std::vector<uint8_t>(slices.begin() + idx * bs + off,
                                            slices.begin() + idx * bs + off + n);
            return p.read_recovery(recs[idx - k], off, n);
        },
        [&](size_t idx, std::vector<uint8_t> bytes) {
            memcpy(slices.data() + idx * bs, bytes.data(), bytes.size());
        });
    g0 = 0;
    for (const FileInfo &f : p.files_in_order) {
        const size_t nb = static_cast<size_t>((f.length + bs - 1) / bs);
        bool touched = false;
        for (size_t b = 0; b < nb; ++b)
            touched = touched || dset.count(g0 + b);
        if (touched) {
            FILE *fh = fopen((fs::path(dir) / f.name).string().c_str(), "wb");
            if (!fh || (f.length && fwrite(slices.data() + g0 * bs, 1, f.length, fh) != f.length))
                return 4;
            fclose(fh);
        }
        g0 += nb;
    }
    printf("repaired %zu\n", damaged.size());
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 3)
        return 2;
    const std::string cmd = argv[1];
    try {
        if (cmd == "parse")
            return cmd_parse(argv[2]);
        if (cmd == "headers" && argc >= 5)
            return cmd_headers(argv[2], std::stoull(argv[3]), argc - 4, argv + 4);
        if (cmd == "create" && argc >= 7)
            return cmd_create(argv[2], std::stoull(argv[3]), std::stof(argv[4]), argv[5], argc - 6,
                              argv + 6);
        if (cmd == "repair" && argc >= 4)
            return cmd_repair(argv[2], argv[3]);
        if (cmd == "volumes" && argc >= 5) {
            std::vector<uint32_t> exps(std::stoul(argv[3]));
            for (size_t e = 0; e < exps.size(); ++e)
                exps[e] = static_cast<uint32_t>(e);
            const VolumeScheme scheme =
                std::string(argv[2]) == "single" ? VolumeScheme::Single : VolumeScheme::Exponential;
            for (const VolumeInfo &v : split_into_volumes(exps, scheme, argv[4]))
                printf("%u %u %zu %s\n", v.exponent_start, v.exponent_end, v.exponents.size(),
                       v.path.string().c_str());
            return 0;
        }
        if (cmd == "volname" && argc >= 6) {
            printf("%s\n", generate_volume_filename(argv[2], std::stoul(argv[3]), std::stoul(argv[4]),
                                                    std::stoul(argv[5]))
                                .c_str());
            return 0;
        }
        if (cmd == "reccount" && argc >= 5) {
            printf("%llu\n", static_cast<unsigned long long>(recovery_block_count(
                                  std::stoull(argv[2]), std::stoull(argv[3]), std::stof(argv[4]))));
            return 0;
        }
        if (cmd == "idless" && argc >= 4) {
            FileHash a{}, b{};
            for (int i = 0; i < 16; ++i) {
                a[i] = static_cast<uint8_t>(std::stoul(std::string(argv[2] + 2 * i, 2), nullptr, 16));
                b[i] = static_cast<uint8_t>(std::stoul(std::string(argv[3] + 2 * i, 2), nullptr, 16));
            }
            printf("%d\n", file_id_less(a, b) ? 1 : 0);
            return 0;
        }
        if (cmd == "padwidth") {
            for (int i = 2; i < argc; ++i)
                printf("%zu\n", calculate_padding_width(std::stoul(argv[i])));
            return 0;
        }
        if (cmd == "blocksize") {
            for (int i = 2; i < argc; ++i)
                printf("%llu\n", static_cast<unsigned long long>(calculate_block_size(std::stoull(argv[i]))));
            return 0;
        }
    } catch (const std::exception &e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 2;
}
