// ZIP archive reading for the asset loaders (host code), over the system
// zlib's raw inflate, with the acceptance rules of the reference loaders'
// archive reader (miniz, vendor/miniz.c in the reference): the end record is
// the last signature with a whole record after it within 64 KiB + 22 bytes of
// the end (searched in 4 KiB windows); data in front of the archive shifts
// its offsets; a stored entry's size test reads the 32-bit word at the
// method field; entries without compressed bytes are empty and unchecked;
// every other payload is CRC-32 checked.  Archives with ZIP64 records are
// rejected.
#pragma once
#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace gs {
namespace zip_detail {
inline uint16_t le16(const uint8_t* p) { return (uint16_t)(p[0] | p[1] << 8); }
inline uint32_t le32(const uint8_t* p) {
    return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}
}  // namespace zip_detail

struct ZipEntry {
    std::string name;                     // raw bytes (may hold NUL)
    uint16_t flags = 0, method = 0;
    uint32_t crc = 0, csize = 0, usize = 0, local = 0, external_attr = 0;
};

struct Zip {
    std::vector<uint8_t> bytes;
    std::vector<ZipEntry> entries;
    size_t base = 0;    // bytes before the archive proper (data in front of it)
    size_t size = 0;    // archive size from `base`

    // Bytes [ofs, ofs + count) of the archive (relative to `base`), or
    // nullptr when the file ends first.
    const uint8_t* at(uint64_t ofs, uint64_t count) const {
        const uint64_t abs = (uint64_t)base + ofs;
        if (abs > bytes.size() || count > bytes.size() - abs) return nullptr;
        return bytes.data() + abs;
    }

    // The end-of-central-directory record: the last signature with a whole
    // record after it, searched backwards in 4 KiB windows (overlapping by 3
    // bytes) until a window starts 64 KiB + 22 bytes or more before the end.
    bool locate_end(size_t& eocd) const {
        using zip_detail::le32;
        const size_t n = bytes.size();
        if (n < 22) return false;
        size_t cur = n > 4096 ? n - 4096 : 0;
        for (;;) {
            const size_t m = std::min<size_t>(4096, n - cur);
            for (long i = (long)m - 4; i >= 0; --i) {
                if (le32(&bytes[cur + (size_t)i]) == 0x06054b50u && n - (cur + (size_t)i) >= 22) {
                    eocd = cur + (size_t)i;
                    return true;
                }
            }
            if (cur == 0 || n - cur >= 65535u + 22u) return false;
            cur = cur > 4093 ? cur - 4093 : 0;
        }
    }

    // Central directory.  Offsets in the archive are relative to its start,
    // which is where the directory's own offset and size say it is: data in
    // front of the archive (the gap between the directory's end and the end
    // record) shifts every offset.
    bool open() {
        using namespace zip_detail;
        size_t eocd;
        if (!locate_end(eocd)) return false;
        const uint8_t* e = &bytes[eocd];
        if (eocd >= 20 + 56 && le32(&bytes[eocd - 20]) == 0x07064b50u) return false;   // ZIP64
        const uint32_t disk = le16(e + 4), cd_disk = le16(e + 6), on_disk = le16(e + 8), total = le16(e + 10);
        const uint32_t cd_size = le32(e + 12), cd_off = le32(e + 16);
        if (total != on_disk) return false;
        if ((disk | cd_disk) != 0 && (disk != 1 || cd_disk != 1)) return false;
        if ((uint64_t)cd_size < (uint64_t)total * 46) return false;
        if ((uint64_t)cd_off + cd_size > bytes.size() || eocd < (uint64_t)cd_off + cd_size) return false;
        base = eocd - ((size_t)cd_off + cd_size);
        size = bytes.size() - base;
        if (!total) return true;
        const uint8_t* cd = at(cd_off, cd_size);
        if (!cd) return false;
        size_t left = cd_size;
        for (uint32_t i = 0; i < total; ++i) {
            if (left < 46 || le32(cd) != 0x02014b50u) return false;
            ZipEntry z;
            z.flags = le16(cd + 8);
            z.method = le16(cd + 10);
            z.crc = le32(cd + 16);
            z.csize = le32(cd + 20);
            z.usize = le32(cd + 24);
            const uint32_t name_len = le16(cd + 28), extra_len = le16(cd + 30), comment_len = le16(cd + 32);
            const uint32_t start_disk = le16(cd + 34);
            z.external_attr = le32(cd + 38);
            z.local = le32(cd + 42);
            if (z.csize == 0xFFFFFFFFu || z.usize == 0xFFFFFFFFu || z.local == 0xFFFFFFFFu) return false;  // ZIP64
            // A stored entry must keep its size, unless the 32-bit word at the
            // method field (method and modification time together) is nonzero;
            // a nonempty entry must have compressed bytes.
            if ((le32(cd + 10) == 0 && z.usize != z.csize) || (z.usize && !z.csize)) return false;
            if (start_disk == 0xFFFF || (start_disk != disk && start_disk != 1)) return false;
            if ((uint64_t)z.local + 30 + z.csize > size) return false;
            if (z.flags & 0x2000u) return false;   // masked local headers
            const size_t header = 46 + (size_t)name_len + extra_len + comment_len;
            if (header > left) return false;
            z.name.assign((const char*)cd + 46, name_len);
            entries.push_back(std::move(z));
            cd += header;
            left -= header;
        }
        return true;
    }

    static bool is_directory(const ZipEntry& z) {
        return (!z.name.empty() && z.name.back() == '/') || (z.external_attr & 0x10u);
    }
    static bool usable(const ZipEntry& z) {
        // not encrypted (traditional or strong), not patch data, stored or deflated
        return !(z.flags & (0x1u | 0x40u | 0x20u)) && (z.method == 0 || z.method == 8);
    }

    // Payload of entry z into out (z.usize bytes), CRC-32 checked.  An entry
    // without compressed bytes is empty and not checked.  A stored entry
    // reads its uncompressed size.
    bool extract(const ZipEntry& z, std::vector<uint8_t>& out) const {
        using namespace zip_detail;
        out.assign(z.usize, 0);
        if (!z.csize) return true;
        const uint8_t* local = at(z.local, 30);
        if (!local || le32(local) != 0x04034b50u) return false;
        const uint64_t data = (uint64_t)z.local + 30 + le16(local + 26) + le16(local + 28);
        if (data + z.csize > size) return false;
        if (z.method == 0) {
            const uint8_t* src = at(data, z.usize);
            if (!src) return false;
            if (z.usize) std::memcpy(out.data(), src, z.usize);
        } else {
            const uint8_t* src = at(data, z.csize);
            if (!src) return false;
            z_stream st{};
            if (inflateInit2(&st, -15) != Z_OK) return false;
            st.next_in = const_cast<Bytef*>(src);
            st.avail_in = z.csize;
            st.next_out = out.data();
            st.avail_out = z.usize;
            const int rc = inflate(&st, Z_FINISH);
            const bool done = rc == Z_STREAM_END && st.total_out == z.usize;
            inflateEnd(&st);
            if (!done) return false;
        }
        const uLong crc = crc32(crc32(0L, Z_NULL, 0), out.data(), (uInt)out.size());
        return (uint32_t)crc == z.crc;
    }
};

}  // namespace gs
