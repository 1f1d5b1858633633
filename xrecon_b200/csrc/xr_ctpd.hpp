// xr_ctpd.hpp -- DICOM-CT-PD projection series reader (host code, no GPU).
//
// The bulk half of the reference's load_projection_stack
// (xrecon/utils/mayo.py:145-170): for every file of a series, parse the
// DICOM Part 10 layout (PS3.10 §7; PS3.5 §7 element encoding, §7.5
// sequences, §8 native pixel data), read the view's angle, source z and
// focal-spot offsets from the DICOM-CT-PD private tags, rescale the stored
// pixels (float32(raw) * float32(slope), then + float32(intercept): the two
// float32 roundings numpy makes for `raw.astype(float32) * slope +
// intercept` with Python-float operands), take every col_stride-th stored
// row and row_stride-th stored column, and write the view transposed to
// [detector row, detector column].  Files are spread over worker threads.
//
// Only the common encodings are taken here: implicit or explicit VR little
// endian, 8/16/32-bit single-frame native pixels, and single-valued tags in
// the forms the Python loader decodes the same way (4-byte raw float32,
// FL, FD, US/SS/UL/SL, DS, IS).  Everything else returns
// XR_ERR_UNSUPPORTED so that the caller's general reader handles (or
// rejects) the series; so does any malformed file.  Every read is bounds
// checked against the file's size.
#pragma once

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

namespace ctpd {

constexpr uint32_t kUndefined = 0xFFFFFFFFu;

constexpr uint16_t vr_code(char a, char b) { return (uint16_t)((uint8_t)a << 8 | (uint8_t)b); }
constexpr uint16_t VR_NONE = 0;
constexpr uint16_t VR_OB = vr_code('O', 'B'), VR_OW = vr_code('O', 'W'), VR_UN = vr_code('U', 'N');
constexpr uint16_t VR_SQ = vr_code('S', 'Q'), VR_US = vr_code('U', 'S'), VR_SS = vr_code('S', 'S');
constexpr uint16_t VR_UL = vr_code('U', 'L'), VR_SL = vr_code('S', 'L'), VR_FL = vr_code('F', 'L');
constexpr uint16_t VR_FD = vr_code('F', 'D'), VR_DS = vr_code('D', 'S'), VR_IS = vr_code('I', 'S');

inline bool long_vr(uint16_t vr) {
    static const char* k[] = {"OB", "OD", "OF", "OL", "OV", "OW", "SQ", "SV", "UC", "UN", "UR", "UT", "UV"};
    for (const char* s : k)
        if (vr == vr_code(s[0], s[1])) return true;
    return false;
}

inline uint32_t tag_of(uint16_t g, uint16_t e) { return (uint32_t)g << 16 | e; }

struct Span {
    const uint8_t* p = nullptr;
    uint32_t n = 0;
    uint16_t vr = VR_NONE;
    bool present = false;
};

// The elements the loader reads.
struct Fields {
    Span rows, cols, spp, frames, bits, stored, pixrep, slope, intercept, pixel;
    Span angle, source_z, shift_z, shift_angle, shift_radius;
};

struct Cur {
    const uint8_t* b;
    size_t pos, end;
    bool u16(uint16_t& v) {
        if (end - pos < 2) return false;
        v = (uint16_t)(b[pos] | b[pos + 1] << 8);
        pos += 2;
        return true;
    }
    bool u32(uint32_t& v) {
        if (end - pos < 4) return false;
        v = (uint32_t)b[pos] | (uint32_t)b[pos + 1] << 8 | (uint32_t)b[pos + 2] << 16 | (uint32_t)b[pos + 3] << 24;
        pos += 4;
        return true;
    }
    bool skip(uint32_t n) {
        if (end - pos < n) return false;
        pos += n;
        return true;
    }
};

// VR of the standard tags read by value in an implicit-VR data set.
inline uint16_t implicit_vr(uint32_t tag) {
    switch (tag) {
    case 0x00280010u: case 0x00280011u: case 0x00280002u: case 0x00280100u:
    case 0x00280101u: case 0x00280102u: case 0x00280103u: return VR_US;
    case 0x00280008u: return VR_IS;
    case 0x00281052u: case 0x00281053u: return VR_DS;
    case 0x7FE00010u: return VR_OW;
    case 0x00080016u: case 0x00080018u: return vr_code('U', 'I');
    case 0x00080060u: case 0x00280004u: return vr_code('C', 'S');
    default: return VR_NONE;
    }
}

// Tag, VR and length of the next element; false on truncation or a VR that
// is not two upper-case letters.
inline bool header(Cur& c, bool explicit_vr, uint32_t& tag, uint16_t& vr, uint32_t& len) {
    uint16_t g, e;
    if (!c.u16(g) || !c.u16(e)) return false;
    tag = tag_of(g, e);
    if (g == 0xFFFE) {
        vr = VR_NONE;
        return c.u32(len);
    }
    if (!explicit_vr) {
        vr = implicit_vr(tag);
        return c.u32(len);
    }
    if (c.end - c.pos < 2) return false;
    char a = (char)c.b[c.pos], b = (char)c.b[c.pos + 1];
    c.pos += 2;
    if (a < 'A' || a > 'Z' || b < 'A' || b > 'Z') return false;
    vr = vr_code(a, b);
    if (long_vr(vr)) {
        uint16_t reserved;
        return c.u16(reserved) && c.u32(len);
    }
    uint16_t l16;
    if (!c.u16(l16)) return false;
    len = l16;
    return true;
}

// Walk the items of an undefined-length sequence to its delimiter.
inline bool skip_items(Cur& c, bool explicit_vr, int depth) {
    if (depth > 32) return false;
    for (;;) {
        uint32_t tag, len;
        uint16_t vr;
        if (!header(c, explicit_vr, tag, vr, len)) return false;
        if (tag == 0xFFFEE0DDu) return true;
        if (tag != 0xFFFEE000u) return false;
        if (len != kUndefined) {
            if (!c.skip(len)) return false;
            continue;
        }
        for (;;) {
            uint32_t t, ln;
            uint16_t v;
            if (!header(c, explicit_vr, t, v, ln)) return false;
            if (t == 0xFFFEE00Du) break;
            if (ln == kUndefined) {
                if (v != VR_SQ && v != VR_UN && v != VR_NONE) return false;
                if (!skip_items(c, explicit_vr && v == VR_SQ, depth + 1)) return false;
            } else if (!c.skip(ln)) {
                return false;
            }
        }
    }
}

inline Span* slot(Fields& f, uint32_t tag) {
    switch (tag) {
    case 0x00280010u: return &f.rows;
    case 0x00280011u: return &f.cols;
    case 0x00280002u: return &f.spp;
    case 0x00280008u: return &f.frames;
    case 0x00280100u: return &f.bits;
    case 0x00280101u: return &f.stored;
    case 0x00280103u: return &f.pixrep;
    case 0x00281053u: return &f.slope;
    case 0x00281052u: return &f.intercept;
    case 0x7FE00010u: return &f.pixel;
    case 0x70311001u: return &f.angle;
    case 0x70311002u: return &f.source_z;
    case 0x7033100Bu: return &f.shift_z;
    case 0x7033100Cu: return &f.shift_angle;
    case 0x7033100Du: return &f.shift_radius;
    default: return nullptr;
    }
}

// Parse one file held in memory; false when it is not a file this reader
// takes.
inline bool parse(const uint8_t* buf, size_t n, Fields& f) {
    if (n < 132 || std::memcmp(buf + 128, "DICM", 4) != 0) return false;
    Cur c{buf, 132, n};
    // file meta group (explicit VR little endian)
    std::string ts;
    bool have_ts = false;
    size_t meta_end = n;
    bool grouped = false;
    {
        Cur m = c;
        uint32_t tag, len;
        uint16_t vr;
        if (!header(m, true, tag, vr, len)) return false;
        if (tag == 0x00020000u) {
            uint32_t glen;
            if (len != 4 || !m.u32(glen) || glen > m.end - m.pos) return false;
            meta_end = m.pos + glen;
            grouped = true;
            c.pos = m.pos;
        }
    }
    Cur m{buf, c.pos, meta_end};
    while (m.pos < m.end) {
        if (grouped && m.end - m.pos < 8) {  // padding at the end of the group
            for (size_t i = m.pos; i < m.end; ++i)
                if (m.b[i]) return false;
            m.pos = m.end;
            break;
        }
        size_t save = m.pos;
        uint32_t tag, len;
        uint16_t vr;
        if (!header(m, true, tag, vr, len)) return false;
        if ((tag >> 16) != 0x0002u) {
            if (grouped) return false;
            m.pos = save;
            break;
        }
        if (len == kUndefined || len > m.end - m.pos) return false;
        if (tag == 0x00020010u) {
            if (vr != vr_code('U', 'I')) return false;
            ts.assign((const char*)m.b + m.pos, len);
            have_ts = true;
        }
        m.pos += len;
    }
    c.pos = m.pos;
    if (!have_ts) return false;
    while (!ts.empty() && (ts.back() == '\0' || ts.back() == ' ')) ts.pop_back();
    bool explicit_vr;
    if (ts == "1.2.840.10008.1.2") explicit_vr = false;
    else if (ts == "1.2.840.10008.1.2.1") explicit_vr = true;
    else return false;
    // data set
    while (c.pos < c.end) {
        if (c.end - c.pos < 8) {
            for (size_t i = c.pos; i < c.end; ++i)
                if (c.b[i]) return false;
            break;
        }
        uint32_t tag, len;
        uint16_t vr;
        if (!header(c, explicit_vr, tag, vr, len)) return false;
        if (len == kUndefined) {
            if (tag == 0x7FE00010u) return false;  // encapsulated pixel data
            if (vr != VR_SQ && vr != VR_UN && vr != VR_NONE) return false;
            if (!skip_items(c, explicit_vr && vr == VR_SQ, 0)) return false;
            continue;
        }
        if (len > c.end - c.pos) return false;
        if (Span* s = slot(f, tag)) {
            s->p = c.b + c.pos;
            s->n = len;
            s->vr = vr;
            s->present = true;
        }
        c.pos += len;
    }
    return true;
}

inline uint32_t le32(const uint8_t* p) {
    return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}

// A decimal string holding one value, [+-]digits[.digits][e[+-]digits]
// padded with spaces, and with NULs when `nul_pad` (DS/IS text; raw bytes
// read as a number take spaces only).  Any other form is left to the
// general reader.
inline bool decimal(const uint8_t* p, uint32_t n, bool integer, bool nul_pad, double& out) {
    uint32_t a = 0, b = n;
    auto pad = [nul_pad](uint8_t ch) { return ch == ' ' || (nul_pad && ch == '\0'); };
    while (a < b && pad(p[a])) ++a;
    while (b > a && pad(p[b - 1])) --b;
    if (b == a || b - a > 64) return false;
    char s[72];
    bool digit = false;
    for (uint32_t i = a; i < b; ++i) {
        char ch = (char)p[i];
        bool ok = (ch >= '0' && ch <= '9') || ch == '+' || ch == '-' ||
                  (!integer && (ch == '.' || ch == 'e' || ch == 'E'));
        if (!ok) return false;
        digit |= ch >= '0' && ch <= '9';
        s[i - a] = ch;
    }
    if (!digit) return false;
    s[b - a] = '\0';
    char* endp = nullptr;
    errno = 0;
    if (integer) {
        long long v = std::strtoll(s, &endp, 10);
        if (*endp || errno) return false;
        out = (double)v;
    } else {
        out = std::strtod(s, &endp);
        if (*endp || errno || !std::isfinite(out)) return false;
    }
    return true;
}

// One number as the Python loader reads it: raw bytes (implicit VR or
// UN/OB/OW) of 4 bytes are a float32, other raw bytes a decimal string;
// typed VRs by type.
inline bool number(const Span& s, double& out) {
    if (s.vr == VR_NONE || s.vr == VR_UN || s.vr == VR_OB || s.vr == VR_OW) {
        if (s.n == 4) {
            uint32_t u = le32(s.p);
            float v;
            std::memcpy(&v, &u, 4);
            out = v;
            return true;
        }
        return decimal(s.p, s.n, false, false, out);
    }
    switch (s.vr) {
    case VR_FL: {
        if (s.n != 4) return false;
        uint32_t u = le32(s.p);
        float v;
        std::memcpy(&v, &u, 4);
        out = v;
        return true;
    }
    case VR_FD: {
        if (s.n != 8) return false;
        uint64_t u = (uint64_t)le32(s.p) | (uint64_t)le32(s.p + 4) << 32;
        std::memcpy(&out, &u, 8);
        return true;
    }
    case VR_US: if (s.n != 2) return false; out = (double)(uint16_t)(s.p[0] | s.p[1] << 8); return true;
    case VR_SS: if (s.n != 2) return false; out = (double)(int16_t)(uint16_t)(s.p[0] | s.p[1] << 8); return true;
    case VR_UL: if (s.n != 4) return false; out = (double)le32(s.p); return true;
    case VR_SL: if (s.n != 4) return false; out = (double)(int32_t)le32(s.p); return true;
    case VR_DS: return decimal(s.p, s.n, false, true, out);
    case VR_IS: return decimal(s.p, s.n, true, true, out);
    default: return false;
    }
}

// A pixel-module integer (US/SS, or IS for the frame count).
inline bool integer(const Span& s, long long& out) {
    double v;
    if (s.vr == VR_US || s.vr == VR_SS || s.vr == VR_IS) {
        if (!number(s, v)) return false;
        out = (long long)v;
        return true;
    }
    return false;
}

struct Job {
    const char* const* paths;
    int nfiles, rows, cols, cs, rs, nv, nu;
    float* sino;
    float* views;
    std::atomic<int> next{0};
    std::atomic<int> failed{-1};
};

template <typename T>
inline void convert(const uint8_t* px, int cols, int cs, int rs, int nv, int nu, float slope, float icpt,
                    int shift, float* out) {
    for (int r = 0; r < nv; ++r) {
        const long long col = (long long)r * rs;
        float* o = out + (size_t)r * nu;
        for (int c = 0; c < nu; ++c) {
            const long long idx = (long long)c * cs * cols + col;
            T raw;
            std::memcpy(&raw, px + idx * (long long)sizeof(T), sizeof(T));
            if (shift) {  // signed values stored in fewer bits: sign-extend
                using U = typename std::make_unsigned<T>::type;
                raw = (T)(U)((U)raw << shift);
                raw = (T)(raw >> shift);
            }
            const float a = (float)raw * slope;
            o[c] = a + icpt;
        }
    }
}

// Load one file into its view slot; false when the file is not taken.
inline bool load_one(Job& j, int i, std::vector<uint8_t>& buf) {
    FILE* fp = std::fopen(j.paths[i], "rb");
    if (!fp) return false;
    bool ok = std::fseek(fp, 0, SEEK_END) == 0;
    long size = ok ? std::ftell(fp) : -1;
    ok = ok && size >= 0 && std::fseek(fp, 0, SEEK_SET) == 0;
    if (ok) {
        buf.resize((size_t)size);
        ok = size == 0 || std::fread(buf.data(), 1, (size_t)size, fp) == (size_t)size;
    }
    std::fclose(fp);
    if (!ok) return false;
    Fields f;
    if (!parse(buf.data(), buf.size(), f)) return false;
    long long rows, cols, bits, spp = 1, frames = 1, pixrep = 0;
    if (!f.rows.present || !f.cols.present || !f.bits.present || !f.pixel.present) return false;
    if (!integer(f.rows, rows) || !integer(f.cols, cols) || !integer(f.bits, bits)) return false;
    if (f.spp.present && !integer(f.spp, spp)) return false;
    if (f.frames.present && !integer(f.frames, frames)) return false;
    if (f.pixrep.present && !integer(f.pixrep, pixrep)) return false;
    if (rows != j.rows || cols != j.cols || spp != 1 || frames != 1) return false;
    if (bits != 8 && bits != 16 && bits != 32) return false;
    if (pixrep != 0 && pixrep != 1) return false;
    long long stored = bits;
    if (f.stored.present && !integer(f.stored, stored)) return false;
    if (stored < 1 || stored > bits) return false;
    const int shift = (pixrep == 1 && stored < bits) ? (int)(bits - stored) : 0;
    if ((unsigned long long)f.pixel.n < (unsigned long long)(rows * cols * (bits / 8))) return false;
    double slope = 1.0, icpt = 0.0;
    if (f.slope.present && !((f.slope.vr == VR_DS || f.slope.vr == VR_IS) && number(f.slope, slope))) return false;
    if (f.intercept.present && !((f.intercept.vr == VR_DS || f.intercept.vr == VR_IS) && number(f.intercept, icpt)))
        return false;
    double v[5] = {0, 0, 0, 0, 0};
    if (!f.angle.present || !number(f.angle, v[0])) return false;
    if (!f.source_z.present || !number(f.source_z, v[1])) return false;
    if (f.shift_z.present && !number(f.shift_z, v[2])) return false;
    if (f.shift_angle.present && !number(f.shift_angle, v[3])) return false;
    if (f.shift_radius.present && !number(f.shift_radius, v[4])) return false;
    float* out = j.sino + (size_t)i * j.nv * j.nu;
    const float s32 = (float)slope, i32 = (float)icpt;
    if (bits == 16) {
        if (pixrep) convert<int16_t>(f.pixel.p, j.cols, j.cs, j.rs, j.nv, j.nu, s32, i32, shift, out);
        else convert<uint16_t>(f.pixel.p, j.cols, j.cs, j.rs, j.nv, j.nu, s32, i32, 0, out);
    } else if (bits == 8) {
        if (pixrep) convert<int8_t>(f.pixel.p, j.cols, j.cs, j.rs, j.nv, j.nu, s32, i32, shift, out);
        else convert<uint8_t>(f.pixel.p, j.cols, j.cs, j.rs, j.nv, j.nu, s32, i32, 0, out);
    } else {
        if (pixrep) convert<int32_t>(f.pixel.p, j.cols, j.cs, j.rs, j.nv, j.nu, s32, i32, shift, out);
        else convert<uint32_t>(f.pixel.p, j.cols, j.cs, j.rs, j.nv, j.nu, s32, i32, 0, out);
    }
    for (int k = 0; k < 5; ++k) j.views[(size_t)i * 5 + k] = (float)v[k];
    return true;
}

inline void worker(Job* j) {
    std::vector<uint8_t> buf;
    for (;;) {
        if (j->failed.load(std::memory_order_relaxed) >= 0) return;
        const int i = j->next.fetch_add(1, std::memory_order_relaxed);
        if (i >= j->nfiles) return;
        if (!load_one(*j, i, buf)) {
            int expect = -1;
            j->failed.compare_exchange_strong(expect, i);
            return;
        }
    }
}

}  // namespace ctpd
