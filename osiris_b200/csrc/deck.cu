// Reader of the reference simulator's Data_Input deck format, and
// osr_create: deck -> device grid -> the reference's start-up state.
//
// Format (compsim/Data_Input.cpp:13-1349, compsim/MIfstream.cpp:8-47): a
// stream of words of printable ASCII (33..126) separated by anything else.
// Every keyword is found by scanning the deck from its first word for an
// exactly equal word; its values are the words that follow, converted as
// atof converts them (the longest numeric prefix, 0 when none).  Arrays are
// "CON v" (constant), "VAR v..." (one value per cell, x fastest, then y,
// then z), "IVAR" (one per i-column) or "KVAR" (one per k-layer); initial
// conditions in INITCOND mode 0 take "k*v" repeat groups (ECLStar,
// compsim/Data_Input.cpp:1941-1975).  Two quirks of the reference that change
// results are kept: JVAR loops on an uninitialised counter in the reference
// and is rejected here, and pseudo-component critical temperatures from the
// Cavett correlation are multiplied by the integer quotient 9/5 = 1
// (compsim/Init_Calcs.cpp:531).  Host code only.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "osiris_b200.h"

namespace {

constexpr double kTimeFactor = 3600.0;  // deck times are hours (TIMECHFACT, compsim/Functions.h:243)
constexpr double kLn10 = 2.302585092994046;
constexpr double kRGas = 8.3144621;     // RGAS, compsim/Functions.h:216

// COMPNAME library (compsim/Data_Input.cpp:653-952): molecular weight
// [g/mol], Tc [K], Pc [Pa], Vc [cm3/mol], acentric factor, parachor, Zc.
// Standard literature constants; the table must match the reference's so
// that decks written for it load unchanged.
struct LibComp {
    const char *name;
    double mw, tc, pc, vc, acf, parachor, zc;
};
const LibComp kLibrary[] = {
    {"C1", 16.043, 190.56, 4599000, 98.6, 0.008, 74.05, 0.2862},
    {"C2", 30.070, 305.32, 4872000, 145.5, 0.0995, 112.91, 0.2793},
    {"C3", 44.096, 369.83, 4248000, 200, 0.1523, 154.03, 0.2763},
    {"iC4", 58.123, 408.14, 3648000, 262.7, 0.1770, 185.32, 0.2824},
    {"nC4", 58.123, 425.12, 3796000, 255, 0.2002, 193.90, 0.2739},
    {"iC5", 72.150, 460.43, 3381000, 305.8, 0.2275, 229.37, 0.2701},
    {"nC5", 72.150, 469.7, 3370000, 313, 0.2515, 236.00, 0.2701},
    {"nC6", 86.177, 507.6, 3025000, 371, 0.3013, 276.71, 0.2659},
    {"nC7", 100.204, 540.2, 2740000, 428, 0.3495, 318.44, 0.2611},
    {"nC8", 114.231, 568.7, 2490000, 486, 0.3996, 359.33, 0.2559},
    {"nC9", 128.258, 594.6, 2290000, 544, 0.4435, 399.57, 0.2520},
    {"nC10", 142.285, 617.7, 2110000, 600, 0.4923, 440.69, 0.2465},
    {"nC11", 156.312, 639, 1949000, 659, 0.5303, 482.00, 0.2419},
    {"nC12", 170.338, 658, 1820000, 716, 0.5764, 522.26, 0.2382},
    {"nC13", 184.365, 675, 1680000, 775, 0.6174, 536.77, 0.2320},
    {"nC14", 198.392, 693, 1570000, 830, 0.6430, 606.05, 0.2262},
    {"nC15", 212.419, 708, 1480000, 889, 0.6863, 647.43, 0.2235},
    {"nC16", 226.446, 723, 1400000, 944, 0.7174, 688.50, 0.2199},
    {"nC17", 240.473, 736, 1340000, 1000, 0.7697, 730.05, 0.2190},
    {"nC18", 254.5, 747, 1270000, 1060, 0.8114, 771.95, 0.2168},
    {"nC19", 268.527, 758, 1210000, 1120, 0.8522, 813.85, 0.2150},
    {"nC20", 282.553, 768, 1160000, 1170, 0.9069, 853.67, 0.2126},
    {"nC21", 296.580, 781.7, 1147000, 1198, 0.9220, 897.64, 0.2114},
    {"nC22", 310.610, 791.8, 1101000, 1253, 0.9550, 939.55, 0.2095},
    {"nC23", 324.630, 801.3, 1059000, 1307, 0.9890, 981.43, 0.2078},
    {"nC24", 338.680, 810.4, 1019000, 1362, 1.0190, 1023.40, 0.2061},
    {"CO2", 44.010, 304.19, 7382000, 94, 0.2276, 82.00, 0.2744},
    {"O2", 31.999, 154.58, 5043000, 73.4, 0.0218, 0.0, 0.2880},
    {"N2", 28.014, 126.1, 3394000, 90.1, 0.0403, 61.12, 0.2917},
    {"H2S", 34.082, 373.53, 8963000, 98.5, 0.0827, 85.50, 0.2843},
    {"SO2", 64.065, 430.75, 7884000, 122, 0.2451, 0.0, 0.2686},
    {"H2", 2.016, 33.18, 1313000, 64.2, 0.2150, 0.0, 0.3053},
    {"H2O", 18.015, 647.13, 22055000, 56, 0.3449, 0.0, 0.2294},
};

// A malformed deck: the reason is kept for osr_deck_error().
struct DeckError {
    std::string what;
};

// The deck as a word stream with the reference's keyword lookup.
class Words {
  public:
    explicit Words(const std::string &text) {
        std::string cur;
        for (char ch : text) {
            const unsigned char u = (unsigned char)ch;
            if (u >= 33 && u <= 126) {
                cur.push_back(ch);
            } else if (!cur.empty()) {
                w_.push_back(cur);
                cur.clear();
            }
        }
        if (!cur.empty()) w_.push_back(cur);
    }
    // position after the first word equal to kw, or -1
    long find(const char *kw) const {
        for (size_t i = 0; i < w_.size(); i++)
            if (w_[i] == kw) return (long)i + 1;
        return -1;
    }
    long need(const char *kw) const {
        long p = find(kw);
        if (p < 0) throw DeckError{std::string("No ") + kw + " keyword in the deck"};
        return p;
    }
    const std::string &at(long p) const {
        if (p < 0 || (size_t)p >= w_.size()) throw DeckError{"deck ends inside a keyword's values"};
        return w_[(size_t)p];
    }
    double num(long p) const { return atof(at(p).c_str()); }  // the reference converts with atof

  private:
    std::vector<std::string> w_;
};

}  // namespace

// Parsed deck values, in the library's cell order (c = i + nx (j + ny k)).
struct osr_deck {
    int nx = 0, ny = 0, nz = 0, pnc = 0, unc = 0, eos = 0, initcond = 3;
    double restemp = 0, wat_ro = 0, wat_mu = 0, sigma = 1, dtmax = 864000.0, lf = 0, re_f = 0, refp = 0, cpor = 0,
           dcpor = 0, dt = 0, total_time = 0;
    int has_cdif = 0;
    double cdif = 0;
    std::vector<double> di, dj, dk, tor, por, fpor, perm, fperm;
    std::vector<double> mw, tc, pc, vc, acf, parachor, zc, kij, swt, sgt;
    std::vector<double> p0, fp0, sw0, fsw0, z0, fz0;  // initial state; z0 [nc][cells]
    std::vector<int> wells_i;                          // [nw][5]
    std::vector<double> wells_f;                       // [nw][nc+6]
    int nwells = 0;
    osr_model model{};
    int nc() const { return pnc + unc; }
    long cells() const { return (long)nx * ny * nz; }
};

namespace {

std::vector<double> grid_array(const Words &W, const char *kw, int nx, int ny, int nz, bool required,
                               double zero_floor, bool floor) {
    long p = W.find(kw);
    if (p < 0) {
        if (required) throw DeckError{std::string("No ") + kw + " keyword in the deck"};
        return {};
    }
    const std::string mode = W.at(p++);
    const long n = (long)nx * ny * nz;
    std::vector<double> a((size_t)n);
    if (mode == "VAR") {
        for (long c = 0; c < n; c++) {
            a[(size_t)c] = W.num(p + c);
            if (floor && a[(size_t)c] == 0) a[(size_t)c] = zero_floor;
        }
    } else if (mode == "CON") {
        const double v = W.num(p);
        for (auto &x : a) x = v;
    } else if (mode == "IVAR") {
        for (long c = 0; c < n; c++) a[(size_t)c] = W.num(p + c % nx);
    } else if (mode == "KVAR") {
        for (long c = 0; c < n; c++) a[(size_t)c] = W.num(p + c / ((long)nx * ny));
    } else {
        throw DeckError{std::string("Incorrect ") + kw + " keyword format (" + mode + ")"};
    }
    return a;
}

std::vector<double> dims(const Words &W, const char *kw, int count) {
    long p = W.need(kw);
    const std::string mode = W.at(p++);
    std::vector<double> a((size_t)count);
    if (mode == "VAR") {
        for (int i = 0; i < count; i++) a[(size_t)i] = W.num(p + i);
    } else if (mode == "CON") {
        for (auto &x : a) x = W.num(p);
    } else {
        throw DeckError{std::string("Incorrect ") + kw + " keyword format"};
    }
    return a;
}

// n values from repeat groups "k*v" or single values (ECLStar)
std::vector<double> ecl_stream(const Words &W, long p, long n) {
    std::vector<double> out;
    out.reserve((size_t)n);
    while ((long)out.size() < n) {
        const std::string &w = W.at(p++);
        const size_t star = w.find('*');
        if (star != std::string::npos) {
            const long k = (long)atof(w.substr(0, star).c_str());
            const double v = atof(w.substr(star + 1).c_str());
            for (long i = 0; i < k; i++) out.push_back(v);
        } else {
            out.push_back(atof(w.c_str()));
        }
    }
    out.resize((size_t)n);
    return out;
}

double scalar_or(const Words &W, const char *kw, double dflt) {
    long p = W.find(kw);
    return p < 0 ? dflt : W.num(p);
}

void parse(const std::string &text, osr_deck &d) {
    Words W(text);
    long p = W.need("GRID");
    d.nx = (int)W.num(p);
    d.ny = (int)W.num(p + 1);
    d.nz = (int)W.num(p + 2);
    if (d.nx < 1 || d.ny < 1 || d.nz < 1) throw DeckError{"GRID dimensions must be positive"};
    p = W.need("NC");
    d.pnc = (int)W.num(p);
    d.unc = (int)W.num(p + 1);
    const int nc = d.nc();
    if (nc < 1 || nc > OSR_MAX_NC || d.pnc < 0 || d.unc < 0) throw DeckError{"NC outside 1..16 components"};
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const long n = d.cells();
    d.restemp = W.num(W.need("RESTEMP")) + 273.15;
    p = W.need("WATERPROPS");
    d.wat_ro = W.num(p);
    d.wat_mu = W.num(p + 1);
    d.di = dims(W, "DI", nx);
    d.dj = dims(W, "DJ", ny);
    d.dk = dims(W, "DK", nz);
    p = W.find("TOR");
    if (p >= 0 && W.at(p) == "JVAR")
        throw DeckError{"JVAR arrays are not supported (the reference's JVAR loop is malformed)"};
    d.tor = grid_array(W, "TOR", nx, ny, nz, false, 0, false);
    if (d.tor.empty()) d.tor.assign((size_t)n, 1.0);
    d.por = grid_array(W, "POR", nx, ny, nz, true, 1e-11, true);
    p = W.find("CDIF");
    d.has_cdif = p >= 0;
    d.cdif = p >= 0 ? W.num(p) : 0.0;
    d.sigma = scalar_or(W, "SIGMA", 1.0);
    d.dtmax = scalar_or(W, "DTMAX", 864000.0);
    d.fpor = grid_array(W, "FPOR", nx, ny, nz, true, 1e-11, true);
    d.lf = W.num(W.need("Lf"));
    d.re_f = W.num(W.need("Re_f"));
    d.perm.clear();
    for (const char *k : {"PERMI", "PERMJ", "PERMK"}) {
        auto a = grid_array(W, k, nx, ny, nz, true, 0, false);
        d.perm.insert(d.perm.end(), a.begin(), a.end());
    }
    d.fperm.clear();
    for (const char *k : {"FPERMI", "FPERMJ", "FPERMK"}) {
        auto a = grid_array(W, k, nx, ny, nz, true, 0, false);
        d.fperm.insert(d.fperm.end(), a.begin(), a.end());
    }
    d.refp = scalar_or(W, "REFP", 0.0);
    d.cpor = scalar_or(W, "CPOR", 0.0);
    d.dcpor = scalar_or(W, "DCPOR", 0.0);
    const std::string m = W.at(W.need("MODEL"));
    if (m != "PR" && m != "SRK") throw DeckError{"Incorrect EOS keyword format"};
    d.eos = m == "PR" ? OSR_EOS_PR : OSR_EOS_SRK;
    for (auto *v : {&d.mw, &d.tc, &d.pc, &d.vc, &d.acf, &d.parachor, &d.zc}) v->assign((size_t)nc, 0.0);
    std::vector<double> sg((size_t)nc, 0.0), tb((size_t)nc, 0.0);
    if (d.unc) {
        const std::pair<const char *, std::vector<double> *> keys[] = {
            {"SG", &sg}, {"TB", &tb}, {"MW", &d.mw}, {"AC", &d.acf}, {"PCRIT", &d.pc}, {"TCRIT", &d.tc},
            {"VCRIT", &d.vc}, {"ZCRIT", &d.zc}};
        for (const auto &kv : keys) {
            long q = W.find(kv.first);
            if (q >= 0)
                for (int i = 0; i < d.unc; i++) (*kv.second)[(size_t)(d.pnc + i)] = W.num(q + i);
        }
        // pseudo-component correlations, compsim/Init_Calcs.cpp:521-545
        for (int i = d.pnc; i < nc; i++) {
            const double Tb = tb[i] * 5 / 9 - 459.67;
            const double API = 141.5 / sg[i] - 131.5;
            const double Tc = 768.071 + 1.7134 * Tb - 1.0834e-3 * Tb * Tb + 3.889e-7 * Tb * Tb * Tb -
                              8.9213e-3 * Tb * API + 5.3095e-6 * Tb * Tb * API + 3.2712e-8 * Tb * Tb * API * API;
            d.tc[i] = 1 * Tc;  // the reference multiplies by the integer quotient 9/5 = 1
            const double Pc = 2.829 + 9.412e-4 * Tb - 3.0475e-6 * Tb * Tb + 1.5184e-9 * Tb * Tb * Tb -
                              2.0876e-5 * Tb * API + 1.1048e-8 * Tb * Tb * API - 4.827e-8 * Tb * API * API +
                              1.395e-10 * Tb * Tb * API * API;
            d.pc[i] = 6897.549353301566 * std::exp(Pc * kLn10);
            d.acf[i] = (3.0 / 7.0) * std::log(d.pc[i] / 101325) / (kLn10 * (d.tc[i] / tb[i] - 1)) - 1;
            const double Zc = 0.2901 - 0.0879 * d.acf[i];
            d.vc[i] = Zc * kRGas * d.tc[i] / d.pc[i];
        }
    }
    p = W.need("COMPNAME");
    for (int i = 0; i < d.pnc; i++) {
        const std::string &nm = W.at(p + i);
        const LibComp *c = nullptr;
        for (const auto &e : kLibrary)
            if (nm == e.name) c = &e;
        if (!c) throw DeckError{"Unknown Component " + nm};
        d.mw[i] = c->mw;
        d.tc[i] = c->tc;
        d.pc[i] = c->pc;
        d.vc[i] = c->vc;
        d.acf[i] = c->acf;
        d.parachor[i] = c->parachor;
        d.zc[i] = c->zc;
    }
    for (const char *kw : {"SWT", "SGT"}) {
        p = W.need(kw);
        const int rows = (int)W.num(p++);
        if (rows < 1) throw DeckError{std::string("Incorrect ") + kw + " keyword format"};
        std::vector<double> &t = kw[1] == 'W' ? d.swt : d.sgt;
        t.resize((size_t)rows * 4);
        for (int i = 0; i < rows * 4; i++) t[(size_t)i] = W.num(p + i);
    }
    d.kij.assign((size_t)nc * nc, 0.0);
    p = W.find("BIC");
    if (p >= 0)
        for (int i = 1; i < nc; i++)
            for (int j = 0; j < i; j++) {
                const double v = W.num(p++);
                d.kij[(size_t)(i * nc + j)] = d.kij[(size_t)(j * nc + i)] = v;
            }
    d.initcond = (int)W.num(W.need("INITCOND"));
    auto fill_comp = [&](std::vector<double> &z, const std::vector<double> &per_cell_nc) {
        // per_cell_nc is [cells][nc] as the deck lists it; z is [nc][cells]
        z.assign((size_t)nc * n, 0.0);
        for (long c = 0; c < n; c++)
            for (int i = 0; i < nc; i++) z[(size_t)(i * n + c)] = per_cell_nc[(size_t)(c * nc + i)];
    };
    if (d.initcond == 0) {
        d.p0 = ecl_stream(W, W.need("IPRESS"), n);
        d.fp0 = ecl_stream(W, W.need("FIPRESS"), n);
        d.sw0 = ecl_stream(W, W.need("IWS"), n);
        d.fsw0 = ecl_stream(W, W.need("FIWS"), n);
        // IGC / FIGC in mode 0 are [nc][cells] streams
        d.z0 = ecl_stream(W, W.need("IGC"), (long)nc * n);
        d.fz0 = ecl_stream(W, W.need("FIGC"), (long)nc * n);
    } else if (d.initcond == 1) {
        auto layers = [&](const char *kw, int per) {
            long q = W.need(kw);
            std::vector<double> v((size_t)nz * per);
            for (int i = 0; i < nz * per; i++) v[(size_t)i] = W.num(q + i);
            return v;
        };
        const long layer = (long)nx * ny;
        auto per_layer = [&](const char *kw) {
            auto v = layers(kw, 1);
            std::vector<double> a((size_t)n);
            for (long c = 0; c < n; c++) a[(size_t)c] = v[(size_t)(c / layer)];
            return a;
        };
        d.p0 = per_layer("IPRESS");
        d.fp0 = per_layer("FIPRESS");
        d.sw0 = per_layer("IWS");
        d.fsw0 = per_layer("FIWS");
        for (int med = 0; med < 2; med++) {
            auto v = layers(med ? "FIGC" : "IGC", nc);
            std::vector<double> cells_nc((size_t)n * nc);
            for (long c = 0; c < n; c++)
                for (int i = 0; i < nc; i++) cells_nc[(size_t)(c * nc + i)] = v[(size_t)((c / layer) * nc + i)];
            fill_comp(med ? d.fz0 : d.z0, cells_nc);
        }
    } else if (d.initcond == 3) {
        d.p0.assign((size_t)n, W.num(W.need("IPRESS")));
        d.fp0.assign((size_t)n, W.num(W.need("FIPRESS")));
        d.sw0.assign((size_t)n, W.num(W.need("IWS")));
        d.fsw0.assign((size_t)n, W.num(W.need("FIWS")));
        for (int med = 0; med < 2; med++) {
            long q = W.need(med ? "FIGC" : "IGC");
            std::vector<double> cells_nc((size_t)n * nc);
            for (long c = 0; c < n; c++)
                for (int i = 0; i < nc; i++) cells_nc[(size_t)(c * nc + i)] = W.num(q + i);
            fill_comp(med ? d.fz0 : d.z0, cells_nc);
        }
    } else {
        throw DeckError{"INITCOND " + std::to_string(d.initcond) + " is not supported"};
    }
    p = W.need("WELLS");
    d.nwells = (int)W.num(p++);
    if (d.nwells < 0) throw DeckError{"Incorrect WELLS keyword format"};
    d.wells_i.assign((size_t)d.nwells * 5, 0);
    d.wells_f.assign((size_t)d.nwells * (nc + 6), 0.0);
    for (int w = 0; w < d.nwells; w++) {
        for (int k = 0; k < 5; k++) d.wells_i[(size_t)(w * 5 + k)] = (int)W.num(p + k) - 1;
        p += 5;
        d.wells_i[(size_t)(w * 5)] += 1;  // the well type is kept as written
        const int t = d.wells_i[(size_t)(w * 5)];
        int cnt, tstart;
        if (t == 3 || t == 8) {
            cnt = nc + 6;
            tstart = nc + 3;
        } else if (t >= 0 && t <= 7) {
            cnt = 6;
            tstart = 3;
        } else {
            throw DeckError{"Incorrect WELL keyword format"};
        }
        for (int j = 0; j < cnt; j++)
            d.wells_f[(size_t)(w * (nc + 6) + j)] = W.num(p + j) * (j > tstart ? kTimeFactor : 1.0);
        p += cnt;
    }
    d.dt = W.num(W.need("DT")) * kTimeFactor;
    d.total_time = W.num(W.need("TOTALT")) * kTimeFactor;
}

void make_model(osr_deck &d) {
    osr_model &m = d.model;
    std::memset(&m, 0, sizeof(m));
    m.nx = d.nx;
    m.ny = d.ny;
    m.nz = d.nz;
    m.nc = d.nc();
    m.eos = d.eos;
    m.restemp = d.restemp;
    m.wat_ro = d.wat_ro;
    m.wat_mu = d.wat_mu;
    m.refp = d.refp;
    m.cpor = d.cpor;
    m.dcpor = d.dcpor;
    m.lf = d.lf;
    m.re_f = d.re_f;
    m.sigma = d.sigma;
    m.has_cdif = d.has_cdif;
    m.cdif = d.cdif;
    m.di = d.di.data();
    m.dj = d.dj.data();
    m.dk = d.dk.data();
    m.por = d.por.data();
    m.fpor = d.fpor.data();
    m.perm = d.perm.data();
    m.fperm = d.fperm.data();
    m.mw = d.mw.data();
    m.tc = d.tc.data();
    m.pc = d.pc.data();
    m.vc = d.vc.data();
    m.acf = d.acf.data();
    m.parachor = d.parachor.data();
    m.zc = d.zc.data();
    m.kij = d.kij.data();
    m.nswt = (int)(d.swt.size() / 4);
    m.nsgt = (int)(d.sgt.size() / 4);
    m.swt = d.swt.data();
    m.sgt = d.sgt.data();
    m.nwells = d.nwells;
    m.wells_i = d.wells_i.empty() ? nullptr : d.wells_i.data();
    m.wells_f = d.wells_f.empty() ? nullptr : d.wells_f.data();
    m.tor = d.tor.data();
    m.dt = d.dt;
}

thread_local std::string g_deck_error;

}  // namespace

extern "C" {

osr_status osr_deck_open(const char *path, osr_deck **out) {
    if (!path || !out) return OSR_ERR_ARG;
    *out = nullptr;
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        g_deck_error = std::string("cannot open ") + path;
        return OSR_ERR_DECK;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    osr_deck *d = new osr_deck();
    try {
        parse(ss.str(), *d);
    } catch (const DeckError &e) {
        g_deck_error = e.what;
        delete d;
        return OSR_ERR_DECK;
    }
    make_model(*d);
    g_deck_error.clear();
    *out = d;
    return OSR_OK;
}

const char *osr_deck_error(void) { return g_deck_error.c_str(); }

osr_status osr_deck_model(const osr_deck *d, osr_model *out) {
    if (!d || !out) return OSR_ERR_ARG;
    *out = d->model;
    return OSR_OK;
}

osr_status osr_deck_initial_state(const osr_deck *d, int medium, const double **p0, const double **sw0,
                                  const double **z0) {
    if (!d || medium < 0 || medium > 1) return OSR_ERR_ARG;
    if (p0) *p0 = medium ? d->fp0.data() : d->p0.data();
    if (sw0) *sw0 = medium ? d->fsw0.data() : d->sw0.data();
    if (z0) *z0 = medium ? d->fz0.data() : d->z0.data();
    return OSR_OK;
}

osr_status osr_deck_times(const osr_deck *d, double *dt, double *total_time, double *dtmax, int *initcond) {
    if (!d) return OSR_ERR_ARG;
    if (dt) *dt = d->dt;
    if (total_time) *total_time = d->total_time;
    if (dtmax) *dtmax = d->dtmax;
    if (initcond) *initcond = d->initcond;
    return OSR_OK;
}

osr_status osr_deck_close(osr_deck *d) {
    delete d;
    return OSR_OK;
}

// The reference's start-up (compsim/PrimeSim.cpp:68-85): the INITCOND state,
// a flash of every cell-medium as AllFlash does it (compsim/Init_Calcs.cpp:
// 949-962; label, compositions, oil and gas saturations from the liquid
// volume fraction and densities from the Z factors, :715-737), then
// UpdateDependencies(true) (compsim/PetscAUX.cpp:500-545): phase control,
// PCoeff, the row layout and the property sweeps.
osr_status osr_create(const char *deck_path, void *stream, osr_grid **out) {
    if (!deck_path || !out) return OSR_ERR_ARG;
    *out = nullptr;
    osr_deck *d = nullptr;
    osr_status st = osr_deck_open(deck_path, &d);
    if (st) return st;
    osr_grid *g = nullptr;
    st = osr_grid_create(&d->model, &g);
    const int nc = d->nc();
    const long n = d->cells();
    std::vector<double> T((size_t)n, d->restemp), L((size_t)n), Zl((size_t)n), Zg((size_t)n);
    std::vector<double> x((size_t)nc * n), y((size_t)nc * n), sat((size_t)3 * n), rho((size_t)2 * n);
    std::vector<signed char> label((size_t)n);
    osr_fluid fl{nc, d->eos, d->tc.data(), d->pc.data(), d->acf.data(), d->kij.data()};
    for (int med = 0; med < 2 && st == OSR_OK; med++) {
        const std::vector<double> &P0 = med ? d->fp0 : d->p0, &Sw = med ? d->fsw0 : d->sw0,
                                  &Z0 = med ? d->fz0 : d->z0;
        osr_flash_out o{};
        o.label = label.data();
        o.L = L.data();
        o.x = x.data();
        o.y = y.data();
        o.Zl = Zl.data();
        o.Zg = Zg.data();
        st = osr_flash_batch_host(&fl, P0.data(), T.data(), Z0.data(), n, &o, stream);
        if (st) break;
        for (long c = 0; c < n; c++) {
            const double liq = Zl[c] * L[c] / (Zl[c] * L[c] + Zg[c] * (1 - L[c]));
            sat[(size_t)c] = Sw[c];
            sat[(size_t)(n + c)] = liq * (1 - Sw[c]);
            sat[(size_t)(2 * n + c)] = (1 - liq) * (1 - Sw[c]);
            rho[(size_t)c] = P0[c] / (Zl[c] * kRGas * T[c]);
            rho[(size_t)(n + c)] = P0[c] / (Zg[c] * kRGas * T[c]);
        }
        st = osr_grid_set_state(g, med, P0.data(), sat.data(), x.data(), y.data(), Z0.data(), label.data(),
                                rho.data());
    }
    if (st == OSR_OK) st = osr_grid_phase_ctrl(g, stream);
    if (st == OSR_OK) st = osr_grid_refresh_layout(g, stream);
    if (st == OSR_OK) st = osr_grid_update_dependencies(g, stream);
    if (st == OSR_OK && cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) st = OSR_ERR_CUDA;
    osr_deck_close(d);
    if (st != OSR_OK) {
        if (g) osr_grid_destroy(g);
        return st;
    }
    *out = g;
    return OSR_OK;
}

}  // extern "C"
