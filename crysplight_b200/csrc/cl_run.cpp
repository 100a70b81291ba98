// cl_run.cpp — `crysplight_run`: CryspLight's run files through the C-ABI
// alone (no Python, no Julia), the counterpart of both of the reference's
// run scripts:
//
//   crysplight_run [--device N] [--data DIR] [--output-root DIR]
//                  [--n-photons N] [--n-events N] [--print-setup] [--no-write]
//                  run.toml ...
//
// A point-source run file (scripts/run_point_source.jl → run_from_config,
// src/config.jl:72-79): load_setup (src/config.jl:27-69) with the materials
// of data/<name>.toml (the run file's ../data, else the package's data
// directory), one cl_run_photons call, the reference's summary lines
// (src/output.jl:36-52), and output/<tag>/light.h5 plus a copy of the run
// file (src/output.jl:10-32).
//
// A gamma campaign (a run file with a [campaign] table;
// scripts/shoot_gammas.jl:19-90): the gamma material from [gamma] density and
// its XCOM table, the gamma stage of every event on the host
// (cl_gamma_events), every deposit's photons in one cl_run_segments call, the
// reference's summary, and output/<tag>/events.h5 plus a copy of the run file.
//
// --print-setup prints the parsed setup as JSON and runs nothing (no GPU
// needed).
#include <cerrno>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <limits.h>
#include <sys/stat.h>
#include <unistd.h>

#include "../../include/crysplight_cuda.h"
#include "cl_h5.hpp"
#include "cl_toml.hpp"

namespace {

using cltoml::Document;
using cltoml::Table;
using cltoml::Value;

// ---- paths ----
std::string dirname_of(const std::string& p)
{
    const size_t k = p.find_last_of('/');
    if (k == std::string::npos) return ".";
    return k == 0 ? "/" : p.substr(0, k);
}
std::string basename_of(const std::string& p)
{
    const size_t k = p.find_last_of('/');
    return k == std::string::npos ? p : p.substr(k + 1);
}
std::string stem_of(const std::string& p)
{
    std::string b = basename_of(p);
    const size_t k = b.find_last_of('.');
    return k == std::string::npos || k == 0 ? b : b.substr(0, k);
}
std::string join(const std::string& a, const std::string& b)
{
    if (!b.empty() && b[0] == '/') return b;
    return a.empty() || a.back() == '/' ? a + b : a + "/" + b;
}
std::string absolute(const std::string& p)
{
    char buf[PATH_MAX];
    if (realpath(p.c_str(), buf)) return buf;
    throw std::runtime_error("no such file: " + p);
}
bool is_dir(const std::string& p)
{
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}
void make_dirs(const std::string& p)
{
    if (p.empty() || is_dir(p)) return;
    make_dirs(dirname_of(p));
    if (mkdir(p.c_str(), 0777) != 0 && errno != EEXIST) throw std::runtime_error("cannot create " + p);
}
void copy_file(const std::string& from, const std::string& to)
{
    std::ifstream i(from, std::ios::binary);
    std::ofstream o(to, std::ios::binary);
    if (!i || !o) throw std::runtime_error("cannot copy " + from + " to " + to);
    o << i.rdbuf();
}
// The package's data directory: <dir of this executable>/../data.
std::string package_data_dir()
{
    char buf[PATH_MAX];
    const ssize_t n = readlink("/proc/self/exe", buf, sizeof buf - 1);
    if (n <= 0) return "data";
    buf[n] = 0;
    return join(dirname_of(dirname_of(buf)), "data");
}

// ---- typed access to the documents ----
const Table& table(const Document& d, const char* name, const std::string& file)
{
    auto it = d.find(name);
    if (it == d.end()) throw std::runtime_error(file + ": missing table [" + name + "]");
    return it->second;
}
const Value* find(const Table& t, const std::string& key)
{
    auto it = t.find(key);
    return it == t.end() ? nullptr : &it->second;
}
const Value& need(const Table& t, const std::string& key, const std::string& where)
{
    const Value* v = find(t, key);
    if (!v) throw std::runtime_error(where + ": missing key '" + key + "'");
    return *v;
}
double num(const Value& v, const std::string& what)
{
    if (!v.is_number()) throw std::runtime_error(what + " must be a number");
    return v.num();
}
int64_t integer(const Value& v, const std::string& what)
{
    if (v.kind != Value::INT) throw std::runtime_error(what + " must be an integer");
    return v.i;
}
std::string str(const Value& v, const std::string& what)
{
    if (v.kind != Value::STR) throw std::runtime_error(what + " must be a string");
    return v.s;
}
std::vector<double> vec3(const Value& v, const std::string& what)
{
    if (v.kind != Value::ARRAY || v.arr.size() != 3) throw std::runtime_error(what + " must be 3 numbers");
    return {num(v.arr[0], what), num(v.arr[1], what), num(v.arr[2], what)};
}

// ---- load_setup, src/config.jl:27-69 ----
struct Setup {
    std::string tag, cfg_path, outdir, crystal_name, wrap_name, finish;
    double sigma_alpha_deg = 0.0;
    cl_box box{};
    cl_optical_params op{};
    cl_readout ro{};
    cl_time_binning tb{};
    float pos[3] = {0, 0, 0};
    float tau_ns = 0.0f;
    int64_t n_photons = 0;
    uint64_t seed = 0;
    int32_t max_bounces = 100000;
};

Document load_material(const std::string& name, const std::string& data_dir)
{
    const std::string path = join(data_dir, name + ".toml");
    std::ifstream probe(path);
    if (!probe) throw std::runtime_error("material file not found: " + path);
    return cltoml::parse_file(path);
}

Setup load_setup(const std::string& cfg_arg, const std::string& data_override, const std::string& out_root)
{
    Setup s;
    s.cfg_path = absolute(cfg_arg);
    const Document cfg = cltoml::parse_file(s.cfg_path);
    const std::string root = dirname_of(dirname_of(s.cfg_path));
    std::string data_dir = data_override;
    if (data_dir.empty()) data_dir = is_dir(join(root, "data")) ? join(root, "data") : package_data_dir();

    const Table& run = table(cfg, "run", s.cfg_path);
    const Value* tag = find(run, "tag");
    s.tag = tag ? str(*tag, "run.tag") : stem_of(s.cfg_path);
    s.crystal_name = str(need(table(cfg, "crystal", s.cfg_path), "material", "[crystal]"), "crystal.material");
    s.wrap_name = str(need(table(cfg, "wrap", s.cfg_path), "material", "[wrap]"), "wrap.material");
    const Table& sipm_cfg = table(cfg, "sipm", s.cfg_path);
    const std::string sipm_name = str(need(sipm_cfg, "material", "[sipm]"), "sipm.material");
    const Document crystal = load_material(s.crystal_name, data_dir);
    const Document wrap = load_material(s.wrap_name, data_dir);
    const Document sipm = load_material(sipm_name, data_dir);
    const Table& C = crystal.at("");
    const Table& W = wrap.at("");
    const Table& S = sipm.at("");

    const std::vector<double> sz = vec3(need(table(cfg, "crystal", s.cfg_path), "size_mm", "[crystal]"),
                                        "crystal.size_mm");
    for (int i = 0; i < 3; ++i) s.box.L[i] = (float)sz[i];

    // OpticalParams, src/config.jl:39-50 (every value rounded once to Float32)
    const Value* pde_o = find(sipm_cfg, "pde_override");
    s.op.pde = (float)num(pde_o ? *pde_o : need(S, "pde", sipm_name), "pde");
    s.op.n_crystal = (float)num(need(C, "n", s.crystal_name), "n");
    s.op.n_coupling = (float)num(need(sipm_cfg, "coupling_n", "[sipm]"), "coupling_n");
    s.op.abs_len_mm = (float)num(need(C, "abs_length_mm", s.crystal_name), "abs_length_mm");
    const Value* ray = find(C, "rayleigh_mm");
    s.op.rayleigh_mm = ray ? (float)num(*ray, "rayleigh_mm") : INFINITY;
    s.op.wrap_R = (float)num(need(W, "reflectivity", s.wrap_name), "reflectivity");
    s.op.wrap_specular = str(need(W, "model", s.wrap_name), "model") == "specular" ? 1 : 0;
    const auto surf_it = cfg.find("surface");
    const Table empty;
    const Table& surf = surf_it == cfg.end() ? empty : surf_it->second;
    const Value* fin = find(surf, "finish");
    s.finish = fin ? str(*fin, "surface.finish") : "backpainted";
    if (s.finish != "backpainted" && s.finish != "frontpainted")
        throw std::runtime_error("unknown finish: " + s.finish);                // src/config.jl:22-25
    s.op.air_gap = s.finish == "backpainted" ? 1 : 0;
    const Value* sa = find(surf, "sigma_alpha_deg");
    s.sigma_alpha_deg = sa ? num(*sa, "surface.sigma_alpha_deg") : 0.0;
    s.op.sigma_alpha = (float)(s.sigma_alpha_deg * (M_PI / 180.0));              // Float32(deg2rad(x))

    s.ro.grid.pitch_mm = (float)num(need(S, "pitch_mm", sipm_name), "pitch_mm");
    s.ro.grid.nx = (int32_t)integer(need(S, "nx", sipm_name), "nx");
    s.ro.grid.ny = (int32_t)integer(need(S, "ny", sipm_name), "ny");

    const Table& bin = table(cfg, "binning", s.cfg_path);
    s.tb.bin_ns = (float)num(need(bin, "bin_ns", "[binning]"), "bin_ns");
    // round(window / bin) with Julia's round (ties to even), in Float64
    s.tb.nbins = (int32_t)std::nearbyint(num(need(bin, "window_ns", "[binning]"), "window_ns") / (double)s.tb.bin_ns);

    const Table& src = table(cfg, "source", s.cfg_path);
    if (str(need(src, "type", "[source]"), "source.type") != "point")
        throw std::runtime_error("only the point source is supported");
    const std::vector<double> p = vec3(need(src, "position_mm", "[source]"), "source.position_mm");
    for (int i = 0; i < 3; ++i) s.pos[i] = (float)p[i];
    const std::string prof = str(need(src, "time_profile", "[source]"), "source.time_profile");
    s.tau_ns = prof == "delta" ? 0.0f : (float)num(need(C, "tau_ns", s.crystal_name), "tau_ns");

    s.n_photons = integer(need(run, "n_photons", "[run]"), "run.n_photons");
    s.seed = (uint64_t)integer(need(run, "seed", "[run]"), "run.seed");
    const Value* mb = find(run, "max_bounces");
    s.max_bounces = mb ? (int32_t)integer(*mb, "run.max_bounces") : 100000;

    const auto out_it = cfg.find("output");
    const Value* od = out_it == cfg.end() ? nullptr : find(out_it->second, "dir");
    s.outdir = join(join(out_root.empty() ? root : out_root, od ? str(*od, "output.dir") : "output"), s.tag);
    return s;
}

// ---- reporting ----
std::string json_str(const std::string& v)
{
    std::string o = "\"";
    for (char c : v) {
        if (c == '"' || c == '\\') { o += '\\'; o += c; }
        else if ((unsigned char)c < 0x20) { char b[8]; std::snprintf(b, sizeof b, "\\u%04x", c); o += b; }
        else o += c;
    }
    return o + "\"";
}
std::string jf(double v)
{
    if (std::isinf(v)) return v > 0 ? "Infinity" : "-Infinity";
    if (std::isnan(v)) return "NaN";
    char b[40];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

void print_setup(const Setup& s)
{
    std::printf("{\"tag\": %s, \"cfg_path\": %s, \"outdir\": %s, \"box\": [%s, %s, %s], ",
                json_str(s.tag).c_str(), json_str(s.cfg_path).c_str(), json_str(s.outdir).c_str(),
                jf(s.box.L[0]).c_str(), jf(s.box.L[1]).c_str(), jf(s.box.L[2]).c_str());
    std::printf("\"op\": {\"n_crystal\": %s, \"n_coupling\": %s, \"abs_len_mm\": %s, \"rayleigh_mm\": %s, "
                "\"wrap_R\": %s, \"wrap_specular\": %d, \"air_gap\": %d, \"sigma_alpha\": %s, \"pde\": %s}, ",
                jf(s.op.n_crystal).c_str(), jf(s.op.n_coupling).c_str(), jf(s.op.abs_len_mm).c_str(),
                jf(s.op.rayleigh_mm).c_str(), jf(s.op.wrap_R).c_str(), s.op.wrap_specular, s.op.air_gap,
                jf(s.op.sigma_alpha).c_str(), jf(s.op.pde).c_str());
    std::printf("\"grid\": [%s, %d, %d], \"tb\": [%s, %d], \"pos\": [%s, %s, %s], \"tau_ns\": %s, "
                "\"n_photons\": %lld, \"seed\": %llu, \"max_bounces\": %d, \"crystal\": %s, \"wrap\": %s, "
                "\"finish\": %s, \"sigma_alpha_deg\": %s}\n",
                jf(s.ro.grid.pitch_mm).c_str(), s.ro.grid.nx, s.ro.grid.ny, jf(s.tb.bin_ns).c_str(), s.tb.nbins,
                jf(s.pos[0]).c_str(), jf(s.pos[1]).c_str(), jf(s.pos[2]).c_str(), jf(s.tau_ns).c_str(),
                (long long)s.n_photons, (unsigned long long)s.seed, s.max_bounces,
                json_str(s.crystal_name).c_str(), json_str(s.wrap_name).c_str(), json_str(s.finish).c_str(),
                jf(s.sigma_alpha_deg).c_str());
}

// The 8-fold symmetry residual of the time-integrated map (src/output.jl:58-62).
double symmetry_residual(const std::vector<uint32_t>& counts, int nx, int ny, int nb)
{
    if (nx != ny) return NAN;
    std::vector<double> m((size_t)nx * ny, 0.0);
    for (int b = 0; b < nb; ++b)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) m[i + (size_t)nx * j] += counts[i + (size_t)nx * (j + (size_t)ny * b)];
    auto at = [&](int i, int j) { return m[i + (size_t)nx * j]; };
    double worst = 0.0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int ri = nx - 1 - i, rj = ny - 1 - j;
            const double s = (at(i, j) + at(ri, j) + at(i, rj) + at(ri, rj) + at(j, i) + at(rj, i) + at(j, ri) +
                              at(rj, ri)) / 8.0;
            worst = std::fmax(worst, std::fabs(at(i, j) - s) / std::fmax(s, 1.0));
        }
    return worst;
}

void write_light_h5(const Setup& s, const std::vector<uint32_t>& counts, const std::vector<float>& first,
                    const cl_counters& c)
{
    using namespace clh5;
    Writer w;
    const uint64_t nx = (uint64_t)s.ro.grid.nx, ny = (uint64_t)s.ro.grid.ny, nb = (uint64_t)s.tb.nbins + 1;
    Dataset dc{"counts", Type::U32, {nx, ny, nb}, Bytes(counts.size() * 4)};
    std::memcpy(dc.raw.data(), counts.data(), dc.raw.size());
    Dataset df{"first_time_ns", Type::F32, {nx, ny}, Bytes(first.size() * 4)};
    std::memcpy(df.raw.data(), first.data(), df.raw.size());
    w.add_dataset(std::move(dc));
    w.add_dataset(std::move(df));
    w.add_attribute(attr_str("tag", s.tag));
    w.add_attribute(attr_num("n_photons", Type::I64, (int64_t)s.n_photons));
    w.add_attribute(attr_num("seed", Type::I64, (int64_t)s.seed));
    w.add_attribute(attr_num("bin_ns", Type::F32, s.tb.bin_ns));
    w.add_attribute(attr_num("nbins", Type::I32, s.tb.nbins));
    w.add_attribute(attr_str("crystal", s.crystal_name));
    w.add_attribute(attr_str("wrap", s.wrap_name));
    w.add_attribute(attr_num("pde", Type::F32, s.op.pde));
    w.add_attribute(attr_num("ndet", Type::I64, c.ndet));
    w.add_attribute(attr_num("nabs_bulk", Type::I64, c.nabs_bulk));
    w.add_attribute(attr_num("nabs_wall", Type::I64, c.nabs_wall));
    w.add_attribute(attr_num("nabs_sipm", Type::I64, c.nabs_sipm));
    w.add_attribute(attr_num("ncap", Type::I64, c.ncap));
    w.add_attribute(attr_num("nabs_surround", Type::I64, c.nabs_sur));
    w.add_attribute(attr_num("nscat", Type::I64, c.nscat));
    w.add_attribute(attr_str("finish", s.finish));
    w.add_attribute(attr_num("sigma_alpha_deg", Type::F64, s.sigma_alpha_deg));
    make_dirs(s.outdir);
    copy_file(s.cfg_path, join(s.outdir, basename_of(s.cfg_path)));
    w.write(join(s.outdir, "light.h5"));
}

int run_one(cl_handle* h, const Setup& s, bool write)
{
    const int nx = s.ro.grid.nx, ny = s.ro.grid.ny, nb = s.tb.nbins + 1;
    std::vector<uint32_t> counts((size_t)nx * ny * nb);
    std::vector<float> first((size_t)nx * ny);
    cl_counters c{};
    const float px = s.pos[0], py = s.pos[1], pz = s.pos[2];
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = cl_run_photons(h, &s.box, &s.op, &s.ro, &s.tb, &px, &py, &pz, nullptr, 1, s.n_photons,
                                  s.seed, 0, s.tau_ns, s.max_bounces, counts.data(), first.data(), &c, nullptr);
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != CL_OK) {
        std::fprintf(stderr, "%s: cl_run_photons failed (%d): %s\n", s.cfg_path.c_str(), rc, cl_last_error(h));
        return 1;
    }
    if (write) write_light_h5(s, counts, first, c);
    const double n = (double)s.n_photons;
    const double mb = c.ndet > 0 ? (double)c.sum_bounces_det / (double)c.ndet : NAN;
    std::printf("%-22s  detected %6.2f%%   bulk %6.2f%%   wall %6.2f%%   cap %.2e\n", s.tag.c_str(),
                100.0 * c.ndet / n, 100.0 * c.nabs_bulk / n, 100.0 * c.nabs_wall / n, c.ncap / n);
    std::printf("%-22s  <bounces|det> %.1f   symmetry residual %.3f   %.2fs (CUDA)\n", "", mb,
                symmetry_residual(counts, nx, ny, nb), elapsed);
    std::fflush(stdout);
    return 0;
}

// ---- gamma campaigns, scripts/shoot_gammas.jl:19-90 ----
struct GammaSetup {
    std::string tag, cfg_path, outdir, crystal_name, xcom_path;
    cl_box box{};
    cl_optical_params op{};
    cl_readout ro{};
    cl_time_binning tb{};
    double yield_per_mev = 0.0, density = 0.0;
    float tau_ns = 0.0f;
    int64_t n_events = 0;
    uint64_t seed = 0;
};

GammaSetup load_gamma_setup(const std::string& cfg_arg, const std::string& data_override,
                            const std::string& out_root)
{
    GammaSetup g;
    g.cfg_path = absolute(cfg_arg);
    const Document cfg = cltoml::parse_file(g.cfg_path);
    const std::string root = dirname_of(dirname_of(g.cfg_path));
    std::string data_dir = data_override;
    if (data_dir.empty()) data_dir = is_dir(join(root, "data")) ? join(root, "data") : package_data_dir();
    const Table& camp = table(cfg, "campaign", g.cfg_path);
    g.tag = str(need(camp, "tag", "[campaign]"), "campaign.tag");
    g.n_events = integer(need(camp, "n_events", "[campaign]"), "campaign.n_events");
    if (g.n_events < 1)
        throw std::runtime_error(g.cfg_path + ": campaign.n_events must be >= 1 (got " +
                                 std::to_string(g.n_events) + ")");
    g.seed = (uint64_t)integer(need(camp, "seed", "[campaign]"), "campaign.seed");
    const Table& crystal_cfg = table(cfg, "crystal", g.cfg_path);
    g.crystal_name = str(need(crystal_cfg, "material", "[crystal]"), "crystal.material");
    const std::string wrap_name = str(need(table(cfg, "wrap", g.cfg_path), "material", "[wrap]"), "wrap.material");
    const Table& sipm_cfg = table(cfg, "sipm", g.cfg_path);
    const std::string sipm_name = str(need(sipm_cfg, "material", "[sipm]"), "sipm.material");
    const Document crystal = load_material(g.crystal_name, data_dir);
    const Document wrap = load_material(wrap_name, data_dir);
    const Document sipm = load_material(sipm_name, data_dir);
    const Table& C = crystal.at("");
    const Table& W = wrap.at("");
    const Table& S = sipm.at("");
    const std::vector<double> sz = vec3(need(crystal_cfg, "size_mm", "[crystal]"), "crystal.size_mm");
    for (int i = 0; i < 3; ++i) g.box.L[i] = (float)sz[i];
    const Table& surf = table(cfg, "surface", g.cfg_path);
    const Value* fin = find(surf, "finish");
    const std::string finish = fin ? str(*fin, "surface.finish") : "backpainted";
    if (finish != "backpainted" && finish != "frontpainted") throw std::runtime_error("unknown finish: " + finish);
    g.op.n_crystal = (float)num(need(C, "n", g.crystal_name), "n");
    g.op.n_coupling = (float)num(need(sipm_cfg, "coupling_n", "[sipm]"), "coupling_n");
    g.op.abs_len_mm = (float)num(need(C, "abs_length_mm", g.crystal_name), "abs_length_mm");
    const Value* ray = find(C, "rayleigh_mm");
    g.op.rayleigh_mm = ray ? (float)num(*ray, "rayleigh_mm") : INFINITY;
    g.op.wrap_R = (float)num(need(W, "reflectivity", wrap_name), "reflectivity");
    g.op.wrap_specular = str(need(W, "model", wrap_name), "model") == "specular" ? 1 : 0;
    g.op.air_gap = finish == "backpainted" ? 1 : 0;
    g.op.sigma_alpha = (float)(num(need(surf, "sigma_alpha_deg", "[surface]"), "surface.sigma_alpha_deg") *
                               (M_PI / 180.0));
    const Value* pde_o = find(sipm_cfg, "pde_override");
    g.op.pde = (float)num(pde_o ? *pde_o : need(S, "pde", sipm_name), "pde");
    g.ro.grid.pitch_mm = (float)num(need(S, "pitch_mm", sipm_name), "pitch_mm");
    g.ro.grid.nx = (int32_t)integer(need(S, "nx", sipm_name), "nx");
    g.ro.grid.ny = (int32_t)integer(need(S, "ny", sipm_name), "ny");
    const Table& bin = table(cfg, "binning", g.cfg_path);
    g.tb.bin_ns = (float)num(need(bin, "bin_ns", "[binning]"), "bin_ns");
    g.tb.nbins = (int32_t)std::nearbyint(num(need(bin, "window_ns", "[binning]"), "window_ns") / (double)g.tb.bin_ns);
    g.yield_per_mev = num(need(C, "yield_per_mev", g.crystal_name), "yield_per_mev");
    g.tau_ns = (float)num(need(C, "tau_ns", g.crystal_name), "tau_ns");
    const Table& gam = table(cfg, "gamma", g.cfg_path);
    g.density = num(need(gam, "density", "[gamma]"), "gamma.density");
    g.xcom_path = join(data_dir, str(need(gam, "xcom", "[gamma]"), "gamma.xcom"));
    g.outdir = join(join(out_root.empty() ? root : out_root, "output"), g.tag);
    return g;
}

void print_gamma_setup(const GammaSetup& g)
{
    std::printf("{\"tag\": %s, \"cfg_path\": %s, \"outdir\": %s, \"box\": [%s, %s, %s], ",
                json_str(g.tag).c_str(), json_str(g.cfg_path).c_str(), json_str(g.outdir).c_str(),
                jf(g.box.L[0]).c_str(), jf(g.box.L[1]).c_str(), jf(g.box.L[2]).c_str());
    std::printf("\"op\": {\"n_crystal\": %s, \"n_coupling\": %s, \"abs_len_mm\": %s, \"rayleigh_mm\": %s, "
                "\"wrap_R\": %s, \"wrap_specular\": %d, \"air_gap\": %d, \"sigma_alpha\": %s, \"pde\": %s}, ",
                jf(g.op.n_crystal).c_str(), jf(g.op.n_coupling).c_str(), jf(g.op.abs_len_mm).c_str(),
                jf(g.op.rayleigh_mm).c_str(), jf(g.op.wrap_R).c_str(), g.op.wrap_specular, g.op.air_gap,
                jf(g.op.sigma_alpha).c_str(), jf(g.op.pde).c_str());
    std::printf("\"grid\": [%s, %d, %d], \"tb\": [%s, %d], \"yield_per_mev\": %s, \"tau_ns\": %s, "
                "\"n_events\": %lld, \"seed\": %llu, \"crystal\": %s, \"density\": %s, \"xcom\": %s}\n",
                jf(g.ro.grid.pitch_mm).c_str(), g.ro.grid.nx, g.ro.grid.ny, jf(g.tb.bin_ns).c_str(), g.tb.nbins,
                jf(g.yield_per_mev).c_str(), jf(g.tau_ns).c_str(), (long long)g.n_events,
                (unsigned long long)g.seed, json_str(g.crystal_name).c_str(), jf(g.density).c_str(),
                json_str(g.xcom_path).c_str());
}

// NIST XCOM table (src/gamma/nist_data.jl:19-35): rows of 8 numbers (E,
// coherent, incoherent, photoelectric, pair nuclear, pair electron, totals);
// other lines are skipped.  Returns the columns E, incoherent, photoelectric,
// pair nuclear, pair electron.
std::vector<std::vector<double>> load_xcom(const std::string& path)
{
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot read XCOM table " + path);
    std::vector<std::vector<double>> cols(5);
    std::string line;
    while (std::getline(f, line)) {
        size_t a = line.find_first_not_of(" \t\r\n\f\v");
        if (a == std::string::npos || line[a] < '0' || line[a] > '9') continue;
        std::vector<std::string> fields;
        size_t p = a;
        while (p < line.size()) {
            const size_t q = line.find_first_of(" \t\r\n\f\v", p);
            fields.push_back(line.substr(p, q == std::string::npos ? std::string::npos : q - p));
            if (q == std::string::npos) break;
            p = line.find_first_not_of(" \t\r\n\f\v", q);
            if (p == std::string::npos) break;
        }
        if (fields.size() < 8) continue;
        double v[8];
        for (int i = 0; i < 8; ++i) {
            char* end = nullptr;
            v[i] = std::strtod(fields[i].c_str(), &end);
            if (end == fields[i].c_str() || *end != 0)
                throw std::runtime_error(path + ": bad number '" + fields[i] + "'");
        }
        cols[0].push_back(v[0]); cols[1].push_back(v[2]); cols[2].push_back(v[3]);
        cols[3].push_back(v[4]); cols[4].push_back(v[5]);
    }
    if (cols[0].empty()) throw std::runtime_error("no XCOM data rows in " + path);
    return cols;
}

const char* INT_TYPE_KEY = "-1 = no interaction, 0 = direct photoelectric, X>=1 = X Compton scatters";

int run_gamma(cl_handle* h, const GammaSetup& g, bool write)
{
    const auto t0 = std::chrono::steady_clock::now();
    const auto xc = load_xcom(g.xcom_path);
    cl_gamma_material* m = nullptr;
    if (cl_gamma_material_create(&m, xc[0].data(), xc[1].data(), xc[2].data(), xc[3].data(), xc[4].data(),
                                 (int32_t)xc[0].size(), g.density) != CL_OK) {
        std::fprintf(stderr, "%s: %s\n", g.cfg_path.c_str(), cl_gamma_last_error());
        return 1;
    }
    const int64_t n = g.n_events;
    std::vector<float> edep(n), xyz1(3 * n), e1(n), xyz2(3 * n), e2(n), er(n);
    std::vector<int8_t> int_type(n);
    std::vector<int16_t> n_int(n);
    int64_t cap = std::max<int64_t>(16, 8 * n), nd = 0;
    std::vector<float> dep_xyz, dep_t;
    std::vector<int32_t> dep_ev;
    std::vector<int64_t> dep_ph;
    for (;;) {
        dep_xyz.assign(3 * cap, 0.0f); dep_t.assign(cap, 0.0f); dep_ev.assign(cap, 0); dep_ph.assign(cap, 0);
        const int rc = cl_gamma_events(m, &g.box, 0, n, g.seed, 0.511, g.yield_per_mev, 0, edep.data(),
                                       xyz1.data(), e1.data(), xyz2.data(), e2.data(), er.data(),
                                       int_type.data(), n_int.data(), cap, dep_xyz.data(), dep_t.data(),
                                       dep_ev.data(), dep_ph.data(), &nd);
        if (rc == CL_OK) break;
        if (nd > cap) { cap = nd; continue; }
        std::fprintf(stderr, "%s: %s\n", g.cfg_path.c_str(), cl_gamma_last_error());
        cl_gamma_material_destroy(m);
        return 1;
    }
    cl_gamma_material_destroy(m);
    const int nx = g.ro.grid.nx, ny = g.ro.grid.ny, cells = nx * ny;
    std::vector<uint32_t> maps((size_t)cells * n, 0u);
    std::vector<float> tmin((size_t)cells * n, INFINITY);
    std::vector<int32_t> npe(n, 0);
    std::vector<int64_t> off(nd + 1, 0);
    for (int64_t i = 0; i < nd; ++i) off[i + 1] = off[i] + dep_ph[i];
    if (nd > 0 && off[nd] > 0) {
        std::vector<float> sx(nd), sy(nd), sz(nd);
        for (int64_t i = 0; i < nd; ++i) { sx[i] = dep_xyz[3 * i]; sy[i] = dep_xyz[3 * i + 1]; sz[i] = dep_xyz[3 * i + 2]; }
        cl_counters c{};
        const int rc = cl_run_segments(h, &g.box, &g.op, &g.ro, &g.tb, sx.data(), sy.data(), sz.data(), dep_t.data(),
                                       off.data(), dep_ev.data(), nd, n, g.seed, 0, g.tau_ns, 100000, maps.data(),
                                       tmin.data(), npe.data(), &c, nullptr);
        if (rc != CL_OK) {
            std::fprintf(stderr, "%s: cl_run_segments failed (%d): %s\n", g.cfg_path.c_str(), rc, cl_last_error(h));
            return 1;
        }
    }
    std::vector<uint16_t> maps16(maps.size());
    for (size_t i = 0; i < maps.size(); ++i) maps16[i] = (uint16_t)(maps[i] & 0xFFFFu);   // UInt16 maps wrap
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (write) {
        using namespace clh5;
        auto raw = [](const void* p, size_t bytes) {
            Bytes b(bytes);
            if (bytes) std::memcpy(b.data(), p, bytes);
            return b;
        };
        const uint64_t un = (uint64_t)n, ux = (uint64_t)nx, uy = (uint64_t)ny;
        Writer w;
        w.add_dataset({"edep_kev", Type::F32, {un}, raw(edep.data(), 4 * n)});
        w.add_dataset({"npe", Type::I32, {un}, raw(npe.data(), 4 * n)});
        w.add_dataset({"maps", Type::U16, {ux, uy, un}, raw(maps16.data(), 2 * maps16.size())});
        w.add_dataset({"tmin_ns", Type::F32, {ux, uy, un}, raw(tmin.data(), 4 * tmin.size())});
        w.add_dataset({"xyz1_mm", Type::F32, {3, un}, raw(xyz1.data(), 12 * n)});
        w.add_dataset({"e1_kev", Type::F32, {un}, raw(e1.data(), 4 * n)});
        w.add_dataset({"xyz2_mm", Type::F32, {3, un}, raw(xyz2.data(), 12 * n)});
        w.add_dataset({"e2_kev", Type::F32, {un}, raw(e2.data(), 4 * n)});
        w.add_dataset({"er_kev", Type::F32, {un}, raw(er.data(), 4 * n)});
        w.add_dataset({"int_type", Type::I8, {un}, raw(int_type.data(), n)});
        w.add_dataset({"n_int", Type::I16, {un}, raw(n_int.data(), 2 * n)});
        w.add_attribute(attr_str("tag", g.tag));
        w.add_attribute(attr_num("n_events", Type::I64, (int64_t)n));
        w.add_attribute(attr_num("seed", Type::I64, (int64_t)g.seed));
        w.add_attribute(attr_str("crystal", g.crystal_name));
        w.add_attribute(attr_num("pde", Type::F32, g.op.pde));
        w.add_attribute(attr_str("backend", "cuda"));
        w.add_attribute(attr_str("int_type_key", INT_TYPE_KEY));
        w.add_attribute(attr_str("tmin_nohit", "Inf"));
        make_dirs(g.outdir);
        copy_file(g.cfg_path, join(g.outdir, basename_of(g.cfg_path)));
        w.write(join(g.outdir, "events.h5"));
    }
    // summary, scripts/shoot_gammas.jl:80-90
    int64_t inter = 0;
    std::vector<double> pe;
    for (int64_t i = 0; i < n; ++i) {
        inter += edep[i] > 0.0f;
        if (edep[i] > 510.0f) pe.push_back((double)npe[i]);
    }
    const double nn = (double)std::max<int64_t>(n, 1);
    std::printf("%-14s %lld events (%.1fs, cuda): interacted %.1f%%, photopeak %.1f%%\n", g.tag.c_str(),
                (long long)n, elapsed, 100.0 * inter / nn, 100.0 * pe.size() / nn);
    if (!pe.empty()) {
        // as the reference: printed for any photopeak event; one event has no
        // sample standard deviation (Julia's std gives NaN)
        double mean = 0.0, var = 0.0;
        for (double v : pe) mean += v;
        mean /= pe.size();
        for (double v : pe) var += (v - mean) * (v - mean);
        if (pe.size() > 1) {
            const double sd = std::sqrt(var / (pe.size() - 1));
            std::printf("%-14s photopeak: %.0f pe mean, FWHM/mean %.2f%% (photostatistics+transport only)\n",
                        "", mean, 235.5 * sd / mean);
        } else {
            std::printf("%-14s photopeak: %.0f pe mean, FWHM/mean NaN%% (photostatistics+transport only)\n",
                        "", mean);
        }
    }
    std::fflush(stdout);
    return 0;
}

// One run file: a point source or a gamma campaign.
struct Job {
    bool gamma = false;
    Setup point;
    GammaSetup campaign;
};

void usage()
{
    std::fprintf(stderr,
                 "usage: crysplight_run [--device N] [--data DIR] [--output-root DIR] [--n-photons N]\n"
                 "                      [--n-events N] [--print-setup] [--no-write] run.toml ...\n");
}

}  // namespace

int main(int argc, char** argv)
{
    int device = 0;
    std::string data_dir, out_root;
    int64_t n_override = -1, ev_override = -1;
    bool print_only = false, write = true;
    std::vector<std::string> files;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto arg = [&](const char* name) -> std::string {
            if (i + 1 >= argc) { std::fprintf(stderr, "%s needs a value\n", name); std::exit(2); }
            return argv[++i];
        };
        // a non-negative decimal integer, or exit 2
        auto count = [&](const char* name) -> long long {
            const std::string v = arg(name);
            char* end = nullptr;
            errno = 0;
            const long long x = std::strtoll(v.c_str(), &end, 10);
            if (v.empty() || *end != 0 || errno != 0 || x < 0) {
                std::fprintf(stderr, "%s needs a non-negative integer, got '%s'\n", name, v.c_str());
                std::exit(2);
            }
            return x;
        };
        if (a == "--device") device = (int)count("--device");
        else if (a == "--data") data_dir = arg("--data");
        else if (a == "--output-root") out_root = arg("--output-root");
        else if (a == "--n-photons") n_override = count("--n-photons");
        else if (a == "--n-events") ev_override = count("--n-events");
        else if (a == "--print-setup") print_only = true;
        else if (a == "--no-write") write = false;
        else if (a == "-h" || a == "--help") { usage(); return 0; }
        else if (!a.empty() && a[0] == '-') { usage(); return 2; }
        else files.push_back(a);
    }
    if (files.empty()) { usage(); return 2; }
    std::vector<Job> jobs;
    try {
        for (const std::string& f : files) {
            Job j;
            j.gamma = cltoml::parse_file(absolute(f)).count("campaign") != 0;
            if (j.gamma) {
                j.campaign = load_gamma_setup(f, data_dir, out_root);
                if (ev_override == 0) throw std::runtime_error("--n-events must be >= 1");
                if (ev_override > 0) j.campaign.n_events = ev_override;
            } else {
                j.point = load_setup(f, data_dir, out_root);
                if (n_override >= 0) j.point.n_photons = n_override;
            }
            jobs.push_back(std::move(j));
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "crysplight_run: %s\n", e.what());
        return 1;
    }
    if (print_only) {
        for (const Job& j : jobs) {
            if (j.gamma) print_gamma_setup(j.campaign);
            else print_setup(j.point);
        }
        return 0;
    }
    cl_handle* h = nullptr;
    if (cl_create(&h, device) != CL_OK) {
        std::fprintf(stderr, "crysplight_run: %s\n", cl_last_error(nullptr));
        return 1;
    }
    int rc = 0;
    try {
        for (const Job& j : jobs) rc |= j.gamma ? run_gamma(h, j.campaign, write) : run_one(h, j.point, write);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "crysplight_run: %s\n", e.what());
        rc = 1;
    }
    cl_destroy(h);
    return rc;
}
