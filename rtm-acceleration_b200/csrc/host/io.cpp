// io.cpp -- the reference's file formats, written from their description
// (reference src/io/velocity_io.cpp and src/io/seismic_io.cpp):
//   velocity : raw little-endian float32 with a "key = value" .hdr sidecar
//              (# comments; nx nz dx dz ox oz layout), zfast or xfast on disk,
//              values in (0, 20000] m/s;
//   shots    : RTMS v1 -- "RTMS", int32 version, nshots, nrec, nt, float dt,
//              two reserved int32, then per shot sx, sz, rx[nrec], rz[nrec],
//              traces[nrec*nt] trace-major; or SEG-Y rev 0/1 (formats 1, 2, 3,
//              5, big-endian, shots grouped by field record, scalco applied);
//   images   : raw float32.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "rtm_b200_engine.hpp"

namespace rtm_b200 {
namespace io {
namespace {

std::string trim(const std::string& s) {
    const auto a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const auto b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

std::vector<char> slurp(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open file: " + path);
    return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

template <typename T>
T le(const char* p) {
    T v;
    std::memcpy(&v, p, sizeof(T));
    return v;
}

uint32_t be32(const unsigned char* p) {
    return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | (uint32_t)p[3];
}
int16_t be16s(const unsigned char* p) { return (int16_t)((uint16_t)p[0] << 8 | (uint16_t)p[1]); }

// IBM System/360 single: sign, base-16 exponent (bias 64), 24-bit fraction.
float ibm_to_float(uint32_t w) {
    if ((w & 0x7fffffffu) == 0) return 0.0f;
    const double frac = (double)(w & 0x00ffffffu) / 16777216.0;
    const int ex = (int)((w >> 24) & 0x7f) - 64;
    const double v = frac * std::pow(16.0, ex);
    return (float)((w >> 31) ? -v : v);
}

float apply_scalco(int32_t c, int16_t sc) {
    if (sc > 0) return (float)c * (float)sc;
    if (sc < 0) return (float)c / (float)(-sc);
    return (float)c;
}

}  // namespace

bool read_header_file(const std::string& path, VelocityHeader& h) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
        const auto hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        const auto eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
        if (k == "nx") h.nx = std::stoi(v);
        else if (k == "nz") h.nz = std::stoi(v);
        else if (k == "dx") h.dx = std::stof(v);
        else if (k == "dz") h.dz = std::stof(v);
        else if (k == "ox") h.ox = std::stof(v);
        else if (k == "oz") h.oz = std::stof(v);
        else if (k == "layout") h.layout = v;
    }
    return true;
}

void write_header_file(const std::string& path, const VelocityHeader& h) {
    std::ofstream f(path);
    if (!f) throw std::runtime_error("cannot write header: " + path);
    f << "# RTM velocity model header\n# data file: float32, little-endian, no header\n";
    f << "nx = " << h.nx << "\nnz = " << h.nz << "\ndx = " << h.dx << "\ndz = " << h.dz << "\nox = " << h.ox
      << "\noz = " << h.oz << "\nlayout = " << h.layout << "   # zfast: v[ix*nz+iz]  |  xfast: v[iz*nx+ix]\n";
}

VelocityModel read_velocity_raw(const std::string& path, const VelocityHeader& h) {
    if (h.nx <= 0 || h.nz <= 0) throw std::runtime_error("velocity nx/nz not set (use a .hdr file or --nx/--nz)");
    if (h.layout != "zfast" && h.layout != "xfast") throw std::runtime_error("layout must be zfast or xfast");
    const std::vector<char> raw = slurp(path);
    const std::size_t n = (std::size_t)h.nx * h.nz;
    if (raw.size() != n * 4)
        throw std::runtime_error("velocity file size mismatch: " + std::to_string(raw.size()) + " bytes, expected " +
                                 std::to_string(n * 4));
    VelocityModel m;
    m.grid.nx = h.nx; m.grid.nz = h.nz; m.grid.dx = h.dx; m.grid.dz = h.dz; m.grid.ox = h.ox; m.grid.oz = h.oz;
    m.v.resize(n);
    for (int ix = 0; ix < h.nx; ++ix)
        for (int iz = 0; iz < h.nz; ++iz) {
            const std::size_t src = h.layout == "zfast" ? (std::size_t)ix * h.nz + iz : (std::size_t)iz * h.nx + ix;
            const float v = le<float>(raw.data() + 4 * src);
            if (!(v > 0.0f) || v > 20000.0f) throw std::runtime_error("velocity model contains a non-physical value");
            m.v[(std::size_t)ix * h.nz + iz] = v;
        }
    return m;
}

void write_velocity_raw(const std::string& path, const VelocityModel& m) { write_raw_floats(path, m.v); }

std::vector<ShotRecord> read_shots_raw(const std::string& path) {
    const std::vector<char> d = slurp(path);
    if (d.size() < 32) throw std::runtime_error("RTMS file truncated: " + path);
    if (std::memcmp(d.data(), "RTMS", 4) != 0) throw std::runtime_error(path + ": not an RTMS file (bad magic)");
    const int version = le<int32_t>(d.data() + 4), nshots = le<int32_t>(d.data() + 8);
    const int nrec = le<int32_t>(d.data() + 12), nt = le<int32_t>(d.data() + 16);
    const float dt = le<float>(d.data() + 20);
    if (version != 1) throw std::runtime_error("unsupported RTMS version");
    if (nshots <= 0 || nrec <= 0 || nt <= 0 || !(dt > 0.0f)) throw std::runtime_error("RTMS header contains invalid values");
    const std::size_t per = 8 + 8 * (std::size_t)nrec + 4 * (std::size_t)nrec * nt;
    std::vector<ShotRecord> shots((std::size_t)nshots);
    std::size_t off = 32;
    for (auto& s : shots) {
        if (off + per > d.size()) throw std::runtime_error("RTMS file truncated: " + path);
        s.sx = le<float>(d.data() + off);
        s.sz = le<float>(d.data() + off + 4);
        s.nt = nt;
        s.dt = dt;
        s.rx.resize((std::size_t)nrec);
        s.rz.resize((std::size_t)nrec);
        s.traces.resize((std::size_t)nrec * nt);
        std::memcpy(s.rx.data(), d.data() + off + 8, 4 * (std::size_t)nrec);
        std::memcpy(s.rz.data(), d.data() + off + 8 + 4 * (std::size_t)nrec, 4 * (std::size_t)nrec);
        std::memcpy(s.traces.data(), d.data() + off + 8 + 8 * (std::size_t)nrec, 4 * (std::size_t)nrec * nt);
        off += per;
    }
    return shots;
}

std::vector<ShotRecord> read_shots_segy(const std::string& path, float src_depth, float rec_depth) {
    const std::vector<char> raw = slurp(path);
    if (raw.size() < 3600) throw std::runtime_error("SEG-Y too short: " + path);
    const auto* d = reinterpret_cast<const unsigned char*>(raw.data());
    const int dt_us = be16s(d + 3200 + 16), ns = be16s(d + 3200 + 20), fmt = be16s(d + 3200 + 24);
    if (ns <= 0) throw std::runtime_error("SEG-Y: invalid samples per trace");
    if (dt_us <= 0) throw std::runtime_error("SEG-Y: invalid sample interval");
    int bps = 0;
    if (fmt == 1 || fmt == 2 || fmt == 5) bps = 4;
    else if (fmt == 3) bps = 2;
    else throw std::runtime_error("SEG-Y sample format " + std::to_string(fmt) + " is not supported (use 1, 2, 3 or 5)");
    const std::size_t tb = 240 + (std::size_t)ns * bps;
    const std::size_t ntr = (raw.size() - 3600) / tb;
    if (ntr == 0) throw std::runtime_error("SEG-Y contains no traces");
    const float dt = (float)dt_us * 1e-6f;
    std::vector<ShotRecord> shots;
    int cur_fldr = 0;
    float cur_sx = 0.0f;
    for (std::size_t i = 0; i < ntr; ++i) {
        const unsigned char* th = d + 3600 + i * tb;
        const int fldr = (int32_t)be32(th + 8);
        const int16_t sc = be16s(th + 70);
        const float sx = apply_scalco((int32_t)be32(th + 72), sc);
        const float gx = apply_scalco((int32_t)be32(th + 80), sc);
        if (shots.empty() || fldr != cur_fldr || (fldr == 0 && sx != cur_sx)) {
            shots.emplace_back();
            shots.back().sx = sx;
            shots.back().sz = src_depth;
            shots.back().nt = ns;
            shots.back().dt = dt;
            cur_fldr = fldr;
            cur_sx = sx;
        }
        ShotRecord& s = shots.back();
        s.rx.push_back(gx);
        s.rz.push_back(rec_depth);
        const unsigned char* b = th + 240;
        for (int k = 0; k < ns; ++k) {
            float v = 0.0f;
            if (fmt == 1) v = ibm_to_float(be32(b + 4 * k));
            else if (fmt == 5) { const uint32_t w = be32(b + 4 * k); std::memcpy(&v, &w, 4); }
            else if (fmt == 2) v = (float)(int32_t)be32(b + 4 * k);
            else v = (float)be16s(b + 2 * k);
            s.traces.push_back(v);
        }
    }
    return shots;
}

std::vector<ShotRecord> read_shots(const std::string& path, float src_depth, float rec_depth) {
    const auto dot = path.find_last_of('.');
    std::string ext = dot == std::string::npos ? "" : path.substr(dot);
    for (auto& c : ext) c = (char)std::tolower((unsigned char)c);
    if (ext == ".sgy" || ext == ".segy") return read_shots_segy(path, src_depth, rec_depth);
    return read_shots_raw(path);
}

void write_shots_raw(const std::string& path, const std::vector<ShotRecord>& shots) {
    if (shots.empty()) throw std::runtime_error("no shots to write");
    const int nrec = shots[0].nrec(), nt = shots[0].nt;
    for (const auto& s : shots)
        if (s.nrec() != nrec || s.nt != nt) throw std::runtime_error("RAW format requires constant nrec and nt");
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write shots: " + path);
    const int32_t hdr[4] = {1, (int32_t)shots.size(), nrec, nt};
    const int32_t reserved[2] = {0, 0};
    f.write("RTMS", 4);
    f.write(reinterpret_cast<const char*>(hdr), sizeof hdr);
    f.write(reinterpret_cast<const char*>(&shots[0].dt), 4);
    f.write(reinterpret_cast<const char*>(reserved), sizeof reserved);
    for (const auto& s : shots) {
        f.write(reinterpret_cast<const char*>(&s.sx), 4);
        f.write(reinterpret_cast<const char*>(&s.sz), 4);
        f.write(reinterpret_cast<const char*>(s.rx.data()), 4 * (std::streamsize)nrec);
        f.write(reinterpret_cast<const char*>(s.rz.data()), 4 * (std::streamsize)nrec);
        f.write(reinterpret_cast<const char*>(s.traces.data()), 4 * (std::streamsize)nrec * nt);
    }
    if (!f) throw std::runtime_error("write failed: " + path);
}

void write_raw_floats(const std::string& path, const std::vector<float>& v) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write: " + path);
    f.write(reinterpret_cast<const char*>(v.data()), 4 * (std::streamsize)v.size());
    if (!f) throw std::runtime_error("write failed: " + path);
}

std::vector<float> read_raw_floats(const std::string& path) {
    const std::vector<char> raw = slurp(path);
    if (raw.size() % 4) throw std::runtime_error("file is not a float32 array: " + path);
    std::vector<float> v(raw.size() / 4);
    std::memcpy(v.data(), raw.data(), raw.size());
    return v;
}

}  // namespace io
}  // namespace rtm_b200
