// eup_bgk3d -- the reference's serial program (CODE/SRC/bgk3d.F90) driven
// through the C ABI of include/eup.h on one B200.
//
// Reads the reference's inputs unchanged: the namelist &parameters of
// bgk.input (CODE/SRC/input.F90:46-61), the obstacle file
// obs.0000.00000000.bin when flag1 = 1 (CODE/SRC/build.obs.F90:147-177) or the
// sphere/column/half column the reference creates when flag1 = 2 (flag2 = 1..3,
// voxelised on the device; written back as obs.0000.00000000.bin when flag3 = 2) and,
// with irestart = 1, restore.00.00.00.bin (CODE/SRC/restore_raw.F90:34-63).
// The boundary preset, a compile-time -D flag in the reference
// (CODE/SRC/build.bcond.F90), is a command-line option.  Writes:
//   probe_g.0000.dat   every icheck: itime, u, v, w, rho at (8lx/20, 9ly/16, lz/2-5)
//                      (CODE/SRC/diagnostic.F90:143, CODE/SRC/probe_global.F90:77, format i8,4e14.6)
//   drag_mem.0000.dat  every icheck: itime, Fx, Fy, Fz, C_d of the FP64 momentum exchange
//   monitor.dat        every icheck: itime and the FP64 means of CODE/SRC/diagno.F90:157
//   prof_i/prof_j/prof_k.0000.dat  every icheck: the lines (1..l, m/2, n/2), (l/2, 1..m, n/2),
//                      (l/2, m/2, 1..n) (CODE/SRC/diagnostic.F90:137-139, prof_*.F90, format i5,4(e14.6,1x))
//   u_med.000.000.000.dat  every icheck: z-plane means of CODE/SRC/varm.F90 (format i5,4(e14.6,1x))
//   drag.0000.dat      with --cv-drag: control-volume drag of CODE/SRC/drag.F90:51-67 (R = 100,
//                      delta = 52..67 step 5), one line "delta itime fluxX fluxY 0" per box
//   save.00.00.00.TTTTTTTT.bin every itsave (CODE/SRC/save_raw.F90:41-78)
//   bgk.perf           loop time and MLUPS (CODE/SRC/finalize.F90:58-124)
//
//   eup_bgk3d [--preset cylinder_inf|freeslip|driven|couette|check2d|channel | --bc f,r,ri,le,u,d]
//             [--precision fp32|fp64|fp16|bf16] [--device N] [--drag-length D] [--cv-drag] [--periodic-init]
//             [--input bgk.input]
// init_v = 0..3 builds the initial state of CODE/SRC/init.F90 (--periodic-init: its -DPERIODIC coordinates).
#include <chrono>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "eup.h"

namespace {

// &parameters ... / : name = value[, value ...]; the first value of a list is used
std::map<std::string, std::string> read_namelist(const std::string& path, std::string* err) {
    std::map<std::string, std::string> kv;
    std::ifstream f(path);
    if (!f) {
        *err = "cannot open " + path;
        return kv;
    }
    std::stringstream ss;
    std::string line;
    while (std::getline(f, line)) {
        const auto bang = line.find('!');
        if (bang != std::string::npos) line = line.substr(0, bang);
        ss << line << '\n';
    }
    std::string text = ss.str();
    for (auto& c : text) c = (char)std::tolower((unsigned char)c);
    const auto start = text.find("&parameters");
    if (start == std::string::npos) {
        *err = "no &parameters group in " + path;
        return kv;
    }
    auto end = text.find('/', start);
    std::string body = text.substr(start + 11, end == std::string::npos ? std::string::npos : end - start - 11);
    size_t pos = 0;
    while (true) {
        const auto eq = body.find('=', pos);
        if (eq == std::string::npos) break;
        size_t ns = eq;
        while (ns > 0 && std::isspace((unsigned char)body[ns - 1])) --ns;
        size_t nb = ns;
        while (nb > 0 && (std::isalnum((unsigned char)body[nb - 1]) || body[nb - 1] == '_')) --nb;
        const std::string name = body.substr(nb, ns - nb);
        size_t vs = eq + 1;
        while (vs < body.size() && std::isspace((unsigned char)body[vs])) ++vs;
        size_t ve = vs;
        while (ve < body.size() && body[ve] != ',' && !std::isspace((unsigned char)body[ve])) ++ve;
        std::string val = body.substr(vs, ve - vs);
        for (auto& c : val)
            if (c == 'd') c = 'e';  // Fortran double-precision exponent
        kv[name] = val;
        pos = ve;
    }
    return kv;
}

// Fortran Ew.d edit descriptor (e14.6): "  0.123456E+01"
std::string fmt_e(double x, int w = 14, int d = 6) {
    char buf[64];
    if (x == 0.0 || !std::isfinite(x)) {
        if (!std::isfinite(x)) std::snprintf(buf, sizeof buf, "%*s", w, "NaN");
        else std::snprintf(buf, sizeof buf, "%*s", w, (std::string(x < 0 ? "-" : "") + "0." + std::string(d, '0') + "E+00").c_str());
        return buf;
    }
    int e = (int)std::floor(std::log10(std::fabs(x))) + 1;
    double m = x / std::pow(10.0, e);
    long long r = std::llround(std::fabs(m) * std::pow(10.0, d));
    if (r >= (long long)std::pow(10.0, d)) {  // rounding carried into a new digit
        r /= 10;
        e += 1;
    }
    std::string digits = std::to_string(r);
    digits = std::string(d - digits.size(), '0') + digits;
    char exp[16];
    std::snprintf(exp, sizeof exp, "E%c%02d", e < 0 ? '-' : '+', std::abs(e));
    const std::string s = std::string(x < 0 ? "-" : "") + "0." + digits + exp;
    std::snprintf(buf, sizeof buf, "%*s", w, s.c_str());
    return buf;
}

int die(const std::string& msg, eup_handle* h = nullptr) {
    std::fprintf(stderr, "eup_bgk3d: %s%s%s\n", msg.c_str(), h ? ": " : "", h ? eup_last_error(h) : "");
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::string input = "bgk.input", preset = "cylinder_inf", prec = "fp32", bcarg;
    int device = 0;
    bool cv_drag = false;
    bool periodic_init = false;  // the reference's -DPERIODIC coordinates in init
    double drag_length = 0.0;
    for (int a = 1; a < argc; ++a) {
        const std::string s = argv[a];
        auto next = [&](void) -> std::string { return a + 1 < argc ? argv[++a] : ""; };
        if (s == "--input") input = next();
        else if (s == "--preset") preset = next();
        else if (s == "--bc") bcarg = next();
        else if (s == "--precision") prec = next();
        else if (s == "--device") device = std::atoi(next().c_str());
        else if (s == "--drag-length") drag_length = std::atof(next().c_str());
        else if (s == "--cv-drag") cv_drag = true;
        else if (s == "--periodic-init") periodic_init = true;
        else return die("unknown option " + s);
    }
    std::string err;
    auto kv = read_namelist(input, &err);
    if (!err.empty()) return die(err);
    auto geti = [&](const char* k, long def) { return kv.count(k) ? std::atol(kv[k].c_str()) : def; };
    auto getd = [&](const char* k, double def) { return kv.count(k) ? std::atof(kv[k].c_str()) : def; };
    const int lx = (int)geti("lx", 0), ly = (int)geti("ly", 0), lz = (int)geti("lz", 0);
    const long itfin = geti("itfin", 0), icheck = geti("icheck", 0), itsave = geti("itsave", 0);
    const long isignal = geti("isignal", 0), irestart = geti("irestart", 0), init_v = geti("init_v", 0);
    // CODE/SRC/input.F90:52-54 defaults: created column, VTK dump (not written here)
    const long flag1 = geti("flag1", 2), flag2 = geti("flag2", 2), flag3 = geti("flag3", 1);
    double u0 = getd("u0", 0.0), u_inflow = 0.0, u00 = 0.0;
    if (lx < 1 || ly < 1 || lz < 1) return die("lx, ly, lz missing from " + input);

    eup_config cfg{};
    cfg.lx = lx; cfg.ly = ly; cfg.lz = lz;
    cfg.svisc = getd("svisc", 0.0);
    // boundary presets of CODE/SRC/build.bcond.F90 (front, rear, right, left, up, down)
    struct P { const char* name; int bc[6]; int kind; };  // kind 1: inlet (u_inflow = u0), 2: lid (u00 = u0)
    const P presets[] = {{"cylinder_inf", {5, 4, 0, 0, 0, 0}, 1}, {"freeslip", {5, 4, 3, 3, 3, 3}, 1},
                         {"check2d", {5, 4, 1, 1, 0, 0}, 1},      {"driven", {1, 1, 1, 1, 2, 1}, 2},
                         {"couette", {0, 0, 0, 0, 2, 1}, 2},      {"channel", {0, 0, 0, 0, 1, 1}, 0}};
    int kind = -1;
    for (const P& p : presets)
        if (preset == p.name) {
            std::memcpy(cfg.bc, p.bc, sizeof cfg.bc);
            kind = p.kind;
        }
    if (!bcarg.empty()) {
        if (std::sscanf(bcarg.c_str(), "%d,%d,%d,%d,%d,%d", &cfg.bc[0], &cfg.bc[1], &cfg.bc[2], &cfg.bc[3], &cfg.bc[4],
                        &cfg.bc[5]) != 6)
            return die("--bc needs six comma-separated flags");
        kind = (cfg.bc[1] == 4) ? 1 : (cfg.bc[4] == 2 ? 2 : 0);
    }
    if (kind < 0) return die("unknown preset " + preset);
    if (kind == 1) { u_inflow = u0; u0 = 0.0; }
    if (kind == 2) { u00 = u0; u0 = 0.0; }
    cfg.u0 = u0; cfg.u_inflow = u_inflow; cfg.u00 = u00;
    cfg.precision = prec == "fp64" ? EUP_FP64 : prec == "fp16" ? EUP_FP16_DEV : prec == "bf16" ? EUP_BF16_DEV : EUP_FP32;
    cfg.device = device;
    cfg.cd_rho0 = 1.0;
    cfg.cd_uref = (u_inflow != 0.0) ? u_inflow : (u00 != 0.0 ? u00 : 1.0);
    cfg.cd_length = drag_length > 0 ? drag_length : 1.0;
    cfg.cd_span = lz;

    eup_handle* h = nullptr;
    if (eup_create(&cfg, &h) != EUP_OK) return die("eup_create", nullptr);
    const size_t L2 = lx + 2, M2 = ly + 2, N2 = lz + 2, cells = L2 * M2 * N2;
    const int eb = (cfg.precision == EUP_FP64) ? 8 : 4;
    std::vector<char> store((size_t)19 * cells * eb);
    void* pops[19];
    for (int q = 0; q < 19; ++q) pops[q] = store.data() + (size_t)q * cells * eb;

    if (flag1 == 1) {
        std::vector<int32_t> obs((size_t)lx * ly * lz);
        int64_t nobs = 0;
        if (eup_read_obs_file("obs.0000.00000000.bin", lx, ly, lz, obs.data(), &nobs) != EUP_OK)
            return die("obstacle file", nullptr);
        if (eup_set_obstacles(h, obs.data()) != EUP_OK) return die("eup_set_obstacles", h);
        std::printf("INFO: num. obs       --> %lld\n", (long long)nobs);
    } else if (flag1 == 2) {
        // CODE/SRC/build.obs.F90:201-441: the shape is voxelised on the device
        if (preset == "check2d") return die("flag1 = 2 with the check2d preset: the reference leaves the radius unset");
        eup_geometry geo;
        const int32_t variant = preset == "cylinder_inf" ? EUP_GEOM_VARIANT_CYLINDER_INF : 0;
        if (eup_geometry_reference((int32_t)flag2, lx, ly, lz, variant, &geo) != EUP_OK)
            return die("eup_geometry_reference", nullptr);
        if (eup_build_obstacles(h, &geo) != EUP_OK) return die("eup_build_obstacles", h);
        int64_t nobs = 0;
        if (eup_get_obstacles(h, nullptr, &nobs) != EUP_OK) return die("eup_get_obstacles", h);
        std::printf("INFO: num. obs       --> %lld\n", (long long)nobs);
    } else if (flag1 != 0) {
        return die("flag1 must be 0, 1 or 2");
    }
    if (flag3 == 2 && flag1 != 0) {  // CODE/SRC/build.obs.F90:506-541, listed on the device
        if (eup_write_obstacles(h, "obs.0000.00000000.bin") != EUP_OK) return die("eup_write_obstacles", h);
        std::printf("INFO: obstacle binary dump obs.0000.00000000.bin\n");
    }
    int64_t itstart = 0;
    if (irestart == 1) {
        if (eup_read_raw_state("restore.00.00.00.bin", lx, ly, lz, eb, pops, &itstart) != EUP_OK)
            return die("restore file", nullptr);
    } else {
        // CODE/SRC/init.F90 with the namelist's init_v, after build_bcond has settled u0
        const int32_t glob[3] = {lx, ly, lz}, start[3] = {0, 0, 0};
        if (eup_init_reference((int32_t)init_v, lx, ly, lz, glob, start, periodic_init ? 1 : 0, cfg.u0, eb, pops) !=
            EUP_OK)
            return die("init", nullptr);
    }
    if (eup_upload(h, pops, eb, itstart) != EUP_OK) return die("eup_upload", h);

    FILE* fprobe = std::fopen("probe_g.0000.dat", "w");
    FILE* fdrag = std::fopen("drag_mem.0000.dat", "w");
    FILE* fmon = std::fopen("monitor.dat", "w");
    FILE* fprof[3] = {std::fopen("prof_i.0000.dat", "w"), std::fopen("prof_j.0000.dat", "w"),
                      std::fopen("prof_k.0000.dat", "w")};
    FILE* fvarm = std::fopen("u_med.000.000.000.dat", "w");
    FILE* fcv = cv_drag ? std::fopen("drag.0000.dat", "w") : nullptr;
    std::vector<double> prof((size_t)4 * std::max(lx, std::max(ly, lz)));
    const int32_t probe[3] = {8 * lx / 20, 9 * ly / 16, lz / 2 - 5};
    const bool probe_ok = probe[0] >= 1 && probe[1] >= 1 && probe[2] >= 1;
    const auto t0 = std::chrono::steady_clock::now();
    double diag_s = 0.0;
    for (long it = itstart; it < itfin;) {
        long next = itfin;
        for (long c : {icheck, itsave, isignal})
            if (c > 0) next = std::min(next, (it / c + 1) * c);
        if (eup_step(h, (int32_t)(next - it)) != EUP_OK) return die("eup_step", h);
        it = next;
        const auto d0 = std::chrono::steady_clock::now();
        if (icheck > 0 && it % icheck == 0) {
            double f[3], mon[5], pr[4] = {0, 0, 0, 0};
            if (eup_get_forces(h, f) != EUP_OK) return die("eup_get_forces", h);
            double cd = 0.0;
            eup_get_cd_series(h, it, 1, &cd);
            if (probe_ok && eup_get_probes(h, 1, probe, pr) != EUP_OK) return die("eup_get_probes", h);
            const int mrc = eup_get_monitor(h, mon);
            if (mrc != EUP_OK) return die("eup_get_monitor", h);
            const double rdv = 1.0 / ((double)lx * ly * lz);
            std::fprintf(fprobe, "%8ld%s %s %s %s\n", it, fmt_e(pr[1]).c_str(), fmt_e(pr[2]).c_str(), fmt_e(pr[3]).c_str(),
                         fmt_e(pr[0]).c_str());
            std::fprintf(fdrag, "%8ld %.15e %.15e %.15e %.15e\n", it, f[0], f[1], f[2], cd);
            std::fprintf(fmon, "%8ld%s %s %s %s %s\n", it, fmt_e(mon[1] * rdv).c_str(), fmt_e(mon[2] * rdv).c_str(),
                         fmt_e(mon[3] * rdv).c_str(), fmt_e(mon[0] * rdv).c_str(), fmt_e(mon[4] * rdv).c_str());
            // prof_i(m/2, n/2), prof_j(l/2, n/2), prof_k(l/2, m/2) and varm: "# t=" header,
            // i5,4(e14.6,1x) rows, two empty records
            const int32_t lc[3][2] = {{ly / 2, lz / 2}, {lx / 2, lz / 2}, {lx / 2, ly / 2}};
            const int32_t len[3] = {lx, ly, lz};
            for (int ax = 0; ax < 3; ++ax) {
                if (lc[ax][0] < 1 || lc[ax][1] < 1) continue;
                if (eup_get_line(h, ax, lc[ax][0], lc[ax][1], prof.data()) != EUP_OK) return die("eup_get_line", h);
                std::fprintf(fprof[ax], "# t=%7ld\n", it);
                for (int t = 0; t < len[ax]; ++t)
                    std::fprintf(fprof[ax], "%5d%s %s %s %s \n", t + 1, fmt_e(prof[4 * t]).c_str(),
                                 fmt_e(prof[4 * t + 1]).c_str(), fmt_e(prof[4 * t + 2]).c_str(),
                                 fmt_e(prof[4 * t + 3]).c_str());
                std::fprintf(fprof[ax], "\n\n");
            }
            if (eup_get_plane_means(h, 2, prof.data()) != EUP_OK) return die("eup_get_plane_means", h);
            std::fprintf(fvarm, "# t=%7ld\n", it);
            for (int k = 0; k < lz; ++k)
                std::fprintf(fvarm, "%5d%s %s %s %s \n", k + 1, fmt_e(prof[4 * k]).c_str(), fmt_e(prof[4 * k + 1]).c_str(),
                             fmt_e(prof[4 * k + 2]).c_str(), fmt_e(prof[4 * k + 3]).c_str());
            std::fprintf(fvarm, "\n\n");
            if (fcv) {
                const int radius = 100;  // hard-wired in CODE/SRC/drag.F90:48
                for (int delta = 52; delta <= 67; delta += 5) {
                    const int32_t box[6] = {lx / 4 - radius - delta, lx / 4 + radius + delta,
                                            ly / 2 - radius - delta, ly / 2 + radius + delta, 1, lz};
                    double fl[2];
                    if (eup_get_cv_drag(h, box, fl) != EUP_OK) return die("eup_get_cv_drag", h);
                    std::fprintf(fcv, "%12d%12ld %.8E %.8E %11d\n", delta, it, fl[0], fl[1], 0);
                }
            }
        }
        if (itsave > 0 && it % itsave == 0) {
            if (eup_download(h, pops, eb) != EUP_OK) return die("eup_download", h);
            char name[64];
            std::snprintf(name, sizeof name, "save.00.00.00.%08ld.bin", it);
            if (eup_write_raw_state(name, lx, ly, lz, eb, (const void* const*)pops, it) != EUP_OK)
                return die("eup_write_raw_state", nullptr);
        }
        if (isignal > 0 && it % isignal == 0) {
            eup_synchronize(h);
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::printf(" Mean   time%s %8ld/%8ld\n", fmt_e(el / (double)(it - itstart)).c_str(), it, itfin);
        }
        diag_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - d0).count();
    }
    eup_synchronize(h);
    const double loop_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    FILE* fp = std::fopen("bgk.perf", "w");
    std::fprintf(fp, "# Run info\n %d %d %d\n # loop   time%s\n # diag   time%s\n", lx, ly, lz, fmt_e(loop_s).c_str(),
                 fmt_e(diag_s).c_str());
    std::fprintf(fp, " # Mlups      %14.6f\n", (double)lx * ly * lz * (double)(itfin - itstart) / loop_s / 1e6);
    std::fclose(fp);
    std::fclose(fprobe);
    std::fclose(fdrag);
    std::fclose(fmon);
    for (FILE* f : fprof) std::fclose(f);
    std::fclose(fvarm);
    if (fcv) std::fclose(fcv);
    eup_destroy(h);
    return 0;
}
