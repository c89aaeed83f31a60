// grabnes -- the recursion path of GRABNES's `grabnes Gendata.in` on the B200 library.
//
//     grabnes [Gendata.in]            run the job, write the reference's output files
//     grabnes --print-job [file]      print the job the input describes (JSON) and exit (no GPU)
//
// Mirrors the reference's driver for the recursion DOS (lanczosKuboCode/Src/grabnes.f90, CalcSelect and
// CalcKubo in calc.F90:13-566, KuboDOS in kubo.F90:276-319): the input keys are read as MIO reads them
// (Src/MIO/input.F90, parser.f90: `Section.Name value` lines, '#' comments, keys matched without case,
// '_' and '-', former names through the alias table, numbers as arithmetic expressions), the cell,
// neighbour search, Hamiltonian and Peierls phases are built on the device, and for every field of the
// sweep (magf.F90:20-146) the recursion and the continued fraction write
//     <prefix>.a0.dat, <prefix>.b0.dat   a_n and b_n, one per line        (kubosubs.F90:140-176)
//     <prefix>.DOS                       E and DOS in units of g0          (kubosubs.F90:247-276)
//     <prefix>.AB                        the norm, then a_n b_n per line
// inside m<m:05>_B<B:.4f>/ when the sweep has more than one field.  Everything on the device goes
// through the C ABI of include/grabnes_gpu.h.  Without Calculate.OnlyDOS the Kubo time evolution follows
// (KuboInterval, KuboCn -> <prefix>.cn.dat; KuboTEvol -> <prefix>.Z2_<step>.dat, <prefix>.AB_<step>.dat).
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/grabnes_gpu.h"

namespace {

const double kPi = 3.14159265358979323846;
// the shell radii and constants shared with grabnes_b200/model.py (gendata_keys.inc)
#define GBN_ALIAS(present, former)
#define GBN_SHELL_RADIUS(r) r,
#define GBN_CONST(name, value)
const double kShellRadius[] = {
#include "gendata_keys.inc"
};
#undef GBN_SHELL_RADIUS
#undef GBN_CONST
#define GBN_SHELL_RADIUS(r)
#define GBN_CONST(name, value) const double k##name = value;
#include "gendata_keys.inc"
#undef GBN_CONST
#define GBN_CONST(name, value)
const double kFluxQuantum = kHPLANCK / kQE;   // h/e

[[noreturn]] void die(const std::string& msg)
{
    fprintf(stderr, "ERROR: %s\n*** PROGRAM ABORTED\n", msg.c_str());
    exit(1);
}

std::string norm_key(const std::string& k)
{
    std::string o;
    for (char ch : k)
        if (ch != '_' && ch != '-') o += (char)tolower((unsigned char)ch);
    return o;
}

// former (section-less) names of the keys read here (lanczosKuboCode/Src/MIO/input_aliases.inc)
#undef GBN_ALIAS
#define GBN_ALIAS(present, former) {present, former},
const char* kAliases[][2] = {
#include "gendata_keys.inc"
};

// ---------------------------------------------------------------------------- values
// A number as the reference's parser reads it: an arithmetic expression with + - * / ** and
// parentheses, Fortran exponents (1.0d-3), and the functions acos asin atan cos sin tan sqrt exp.
class Expr {
public:
    explicit Expr(const std::string& s) : s_(s), i_(0) {}
    double eval()
    {
        const double v = sum();
        skip();
        if (i_ != s_.size()) throw std::runtime_error("unexpected '" + s_.substr(i_) + "'");
        return v;
    }

private:
    std::string s_;
    size_t i_;
    void skip()
    {
        while (i_ < s_.size() && isspace((unsigned char)s_[i_])) ++i_;
    }
    bool eat(const char* tok)
    {
        skip();
        const size_t n = strlen(tok);
        if (s_.compare(i_, n, tok) == 0) {
            i_ += n;
            return true;
        }
        return false;
    }
    double sum()
    {
        double v = product();
        for (;;) {
            if (eat("+")) v += product();
            else if (eat("-")) v -= product();
            else return v;
        }
    }
    double product()
    {
        double v = power();
        for (;;) {
            skip();
            if (s_.compare(i_, 2, "**") == 0) return v;   // handled by power()
            if (eat("*")) v *= power();
            else if (eat("/")) v /= power();
            else return v;
        }
    }
    double power()
    {
        const double b = unary();
        if (eat("**")) return pow(b, power());   // right-associative
        return b;
    }
    double unary()
    {
        if (eat("-")) return -unary();
        if (eat("+")) return unary();
        return primary();
    }
    double primary()
    {
        skip();
        if (eat("(")) {
            const double v = sum();
            if (!eat(")")) throw std::runtime_error("missing ')'");
            return v;
        }
        static const char* fn[] = {"acos", "asin", "atan", "cos", "sin", "tan", "sqrt", "exp"};
        for (int k = 0; k < 8; ++k) {
            const size_t n = strlen(fn[k]);
            if (s_.compare(i_, n, fn[k]) == 0 && i_ + n < s_.size() && s_[i_ + n] == '(') {
                i_ += n + 1;
                const double x = sum();
                if (!eat(")")) throw std::runtime_error("missing ')'");
                switch (k) {
                    case 0: return acos(x);
                    case 1: return asin(x);
                    case 2: return atan(x);
                    case 3: return cos(x);
                    case 4: return sin(x);
                    case 5: return tan(x);
                    case 6: return sqrt(x);
                    default: return exp(x);
                }
            }
        }
        // number: digits, optional point, optional exponent e/E/d/D
        std::string num;
        while (i_ < s_.size() && (isdigit((unsigned char)s_[i_]) || s_[i_] == '.')) num += s_[i_++];
        if (num.empty()) throw std::runtime_error("number expected at '" + s_.substr(i_) + "'");
        if (i_ < s_.size() && strchr("eEdD", s_[i_])) {
            size_t j = i_ + 1;
            std::string ex = "e";
            if (j < s_.size() && (s_[j] == '+' || s_[j] == '-')) ex += s_[j++];
            if (j < s_.size() && isdigit((unsigned char)s_[j])) {
                while (j < s_.size() && isdigit((unsigned char)s_[j])) ex += s_[j++];
                num += ex;
                i_ = j;
            }
        }
        return strtod(num.c_str(), nullptr);
    }
};

std::vector<std::string> split_ws(const std::string& s)
{
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && isspace((unsigned char)s[i])) ++i;
        size_t j = i;
        while (j < s.size() && !isspace((unsigned char)s[j])) ++j;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}

class Input {
public:
    void load(const std::string& path)
    {
        FILE* f = fopen(path.c_str(), "r");
        if (!f) die("cannot open input file " + path + ": " + strerror(errno));
        char buf[4096];
        bool in_block = false;
        while (fgets(buf, sizeof buf, f)) {
            std::string line(buf);
            const size_t hash = line.find('#');
            if (hash != std::string::npos) line.resize(hash);
            std::vector<std::string> w = split_ws(line);
            if (w.empty()) continue;
            const std::string k0 = norm_key(w[0]);
            if (k0 == "%block") { in_block = true; continue; }
            if (k0 == "%endblock") { in_block = false; continue; }
            if (in_block) continue;
            std::string val;
            for (size_t i = 1; i < w.size(); ++i) val += (i > 1 ? " " : "") + w[i];
            kv_.emplace(k0, val);   // the first occurrence of a key wins
        }
        fclose(f);
    }
    bool find(const std::string& name, std::string* val) const
    {
        auto it = kv_.find(norm_key(name));
        if (it == kv_.end())
            for (auto& a : kAliases)
                if (norm_key(a[0]) == norm_key(name)) it = kv_.find(norm_key(a[1]));
        if (it == kv_.end()) return false;
        if (val) *val = it->second;
        return true;
    }
    bool has(const std::string& name) const { return find(name, nullptr); }
    double d(const std::string& name, double def, int elem = 0) const
    {
        std::string v;
        if (!find(name, &v)) return def;
        std::vector<std::string> w = split_ws(v);
        if ((int)w.size() <= elem) die("input key " + name + " has too few values");
        try {
            return Expr(w[elem]).eval();
        } catch (const std::exception& e) {
            die("input key " + name + ": " + e.what());
        }
    }
    int count(const std::string& name) const
    {
        std::string v;
        return find(name, &v) ? (int)split_ws(v).size() : 0;
    }
    long i(const std::string& name, long def, int elem = 0) const
    {
        const double v = d(name, (double)def, elem);
        if (v != floor(v)) die("input key " + name + " must be an integer");
        return (long)v;
    }
    bool l(const std::string& name, bool def) const
    {
        std::string v;
        if (!find(name, &v)) return def;
        std::string t;
        for (char ch : split_ws(v).empty() ? std::string() : split_ws(v)[0]) t += (char)tolower((unsigned char)ch);
        if (t == ".true." || t == "true" || t == "t" || t == "yes" || t == ".t.") return true;
        if (t == ".false." || t == "false" || t == "f" || t == "no" || t == ".f.") return false;
        die("input key " + name + " must be a logical, not '" + v + "'");
    }
    std::string s(const std::string& name, const std::string& def) const
    {
        std::string v;
        if (!find(name, &v)) return def;
        std::vector<std::string> w = split_ws(v);
        return w.empty() ? def : w[0];
    }

private:
    std::map<std::string, std::string> kv_;
};

std::string lower(std::string s)
{
    for (auto& ch : s) ch = (char)tolower((unsigned char)ch);
    return s;
}

// ---------------------------------------------------------------------------- the job
struct Job {
    gbn_cell cell{};
    gbn_model model{};
    double g0 = 0, cut2intra = 0, cut2inter = 0;
    bool second_layer = false, moire = false;
    int nrecurs = 0, n_en = 0, seed = 0;
    double eta = 0, emin = 0, emax = 0;   // units of g0
    bool only_dos = false, polynomials = false;
    int npol = 100, nt = 500, nwr = 10;
    double dt = 5.0;   // units of hbar / g0
    int tevol_vectors = 1;   // random-phase vectors of the time evolution (Kubo.TEvolVectors)
    long mbi = 0, mbf = 0, mstep = 1;
    bool field_by_value = false, field_steps_by_value = false;
    double b_value = 0, b_init = 0, b_final = 0, b_step = 0;
    std::string prefix;
    // Haldane term (HamHopHaldane, ham.F90:7043-7142) and its phase sweep (HaldPhaseInit, magf.F90:148-211)
    bool haldane = false, hal_paper = false, hal_opposite = false, hal_setfluxq = false;
    int hal_mode = 0;            // 0 none, 1 Haldane.SpecifyFlux, 2 SpecifyPhase, 3 SpecifyRange
    double hal_t2 = 0.0, hal_flux = 0.0, hal_phase = 0.0;   // t2 in g0
    uint32_t hal_mask = 0;       // Haldane.LayerControl: bit l-1 = layer l of HaldaneLayers
    long mphii = 0, mphif = 0, mphistep = 1;
    bool write_data = false;    // Output.WriteDataFiles
    bool read_data = false;     // Output.ReadDataFiles
    bool read_details = false;  // Neigh.ReadDetails
    gbn_pdos pdos{};        // Kubo.PDOS selection (mode 0: the DOS of the whole cell)
    int seed_set = 1235;    // Kubo.SeedSet: the stream of the layer start vectors
    // moireBLShift.Calc: 0 off (the shifts stay 0), 1 Moire.BLShiftDefinedValues, 2 Moire.BLShiftRange
    int bl_mode = 0, bl_steps = 0;
    double bl_val[4] = {0, 0, 0, 0}, bl_min[4] = {0, 0, 0, 0}, bl_max[4] = {0, 0, 0, 0};
};

Job job_from_input(const Input& in)
{
    Job j;
    const double aG = in.d("Structure.LatticeParameter", 2.46);
    const std::string system = in.s("Run.TypeOfSystem", "Graphene");
    const bool encapsulated = lower(system) == "moireencapsulatedbilayerbasedonmoirecell";
    if (lower(system) == "graphene") j.cell.kind = GBN_CELL_GRAPHENE;
    else if (lower(system) == "twistedbilayerbasedonmoirecell" || encapsulated) j.cell.kind = GBN_CELL_TBG_MOIRE;
    else die("Run.TypeOfSystem " + system + " is not on the recursion path of this program");
    // Structure.TwistedBLAddShift (atoms.F90:352-366)
    if (in.l("Structure.TwistedBLAddShift", false)) {
        if (in.l("Structure.BernalShift", false)) j.cell.add_shift = 1;
        else if (in.l("Structure.BridgeShift", false)) j.cell.add_shift = 2;
        else die("TwistedBLAddShift needs BernalShift or BridgeShift to say which shift is added");
        j.cell.shift_factor = in.d("Structure.BilayerShiftFactor", 0.0);
    }
    if (!in.l("Kubo.Calc", true)) die("this program runs the recursion (Kubo.Calc .true.) only");
    if (in.l("Diag.Calc", false)) die("exact diagonalisation (Diag.Calc) is not part of this program");
    j.cell.aG = aG;
    j.cell.cell_size = (int32_t)in.i("Structure.CellSize", 50);
    j.cell.super_cell = (int32_t)in.i("Structure.SuperCell", 1);
    for (int k = 0; k < 4; ++k) j.cell.m[k] = in.has("Structure.MoireCellParameters")
                                               ? (int32_t)in.i("Structure.MoireCellParameters", 0, k) : 0;
    j.cell.height = in.d("Structure.CellHeight", 40.0);
    j.cell.d_interlayer = in.d("Structure.InterlayerDistance", 3.35);
    j.g0 = in.d("TB.Hopping", -3.72 * aG + 12.14);
    const long tbnn = in.i("TB.NeighLevels", 1);
    if (tbnn < 1 || tbnn > 8) die("TB.NeighLevels must be between 1 and 8");
    const double acc = aG / sqrt(3.0);
    const double r = 0.5 * (kShellRadius[tbnn - 1] + kShellRadius[tbnn]) * acc;
    j.cut2intra = r * r;
    if (in.i("Neigh.LayerNeighbors", 0) != 0) {
        const double x = aG / sqrt(3.0) * 1.1 * in.d("Neigh.LayerDistFactor", 1.0);
        j.cut2inter = x * x;
    } else {
        j.cut2inter = 1.0;
    }
    gbn_model& m = j.model;
    const double g0 = j.g0;
    m.aG = aG;
    m.tbnn = (int32_t)tbnn;
    for (int k = 0; k < tbnn; ++k) {
        m.nradii[k] = kShellRadius[k] * aG / sqrt(3.0) * 1.1;
        m.gn_cc[k] = (k == 0) ? g0 / g0 : 0.0;
    }
    const std::string bl = in.s("Interlayer.TypeOfBL", "None");
    const bool koshino_intra = in.l("Intralayer.KoshinoIntralayer", false);
    if ((bl == "Koshino" || bl == "Mayou" || bl == "HTC") && !koshino_intra) {
        static const double f2g2[8] = {0, 0, -0.2354, 0.1877, 0.0, -0.0633, 0.0, 0.0};   // ham.F90:8331-8350 [eV]
        m.intralayer = 1;
        for (int k = 2; k < 8; ++k) m.tksl[k] = f2g2[k] / g0;
    }
    j.moire = in.l("Moire.Potential", false) && in.l("Moire.Jeil", false);
    if (j.moire) {
        if (in.l("Moire.OnlyH0", false)) m.moire_onsite = 2;
        else if (in.l("Moire.OnlyHZ", false)) m.moire_onsite = 3;
        else if (in.l("Moire.NoH0AndHZ", false)) m.moire_onsite = 4;
        else if (in.l("Moire.H0AndHZ", false)) m.moire_onsite = 1;
        else die("the moire potential needs one of MoireH0AndHZ, MoireOnlyH0, MoireOnlyHZ, MoireNoH0AndHZ");
    }
    const double pref = in.d("Moire.PreFactor", 1.0);
    m.C0 = in.d("Moire.PotC0", -0.01013) / g0 * pref;
    m.Cz = in.d("Moire.PotCz", -0.00901) / g0 * pref;
    m.Phi0 = in.d("Moire.PotPhi0", 1.510233401750693);
    m.Phiz = in.d("Moire.PotPhiz", 0.147131255943122);
    m.Cab = in.d("Moire.PotCab", 0.01134) / g0;
    m.Phiab = in.d("Moire.PotPhiab", 0.342084533390889);
    m.eps = in.d("Moire.LatticePercent", -0.018181818181818);
    m.moire_twisted = in.l("Moire.Twisted", false) ? 1 : 0;
    m.twist_rad = in.d("Moire.TwistAngle", 0.0) * kPi / 180.0;
    m.moire_offdiag = in.l("Moire.OffDiag", false) ? 1 : 0;
    m.moire_mid = (in.l("Moire.OffDiagMidpoint", false) && m.moire_offdiag) ? 1 : 0;
    m.shift1 = in.d("Moire.LayerShift1", 0.0);
    m.sign1 = in.d("Moire.FirstMoireMassFactor", 1.0);
    m.sign2 = in.d("Moire.SecondMoireMassFactor", 1.0);
    // Moire.AddSecondMoire (ham.F90:2652-2704 on-site, 5859-5888 and 7745-7880 bonds)
    m.second_moire = in.l("Moire.AddSecondMoire", false) ? 1 : 0;
    if (m.second_moire && in.l("Structure.BasedOnMoireCellParameters", false))
        die("Moire.AddSecondMoire with Structure.BasedOnMoireCellParameters: the reference's second moire then "
            "reads a lattice mismatch it never sets");
    m.eps_factor = in.d("Moire.LatticePercentFactor", 1.0);
    m.twisted2 = in.l("Moire.Twisted2", false) ? 1 : 0;
    m.twist2_rad = in.d("Moire.TwistAngle2", 0.0) * kPi / 180.0;
    m.rotate_first = in.l("Moire.SecondMoireRotateFirst", true) ? 1 : 0;
    m.shift2 = in.d("Moire.LayerShift2", 0.0);
    {
        const double phi2m = atan((1.0 + m.eps) * sin(m.twist2_rad) / ((1.0 + m.eps) * cos(m.twist2_rad) - 1.0));
        m.shift2_x = m.shift2 * cos(phi2m);
        m.shift2_y = m.shift2 * sin(phi2m);
    }
    // MoireEncapsulatedBilayerBasedOnMoireCell (ham.F90:2607-2640, 5729-5780, 6455-6500)
    m.encapsulated = encapsulated ? 1 : 0;
    m.bl_bottom_rad = in.d("Moire.BilayerBottomAngle", 0.0) * kPi / 180.0;
    m.bl_top_rad = in.d("Moire.BilayerTopAngle", 0.0) * kPi / 180.0;
    m.deact_upper = in.l("Moire.BLDeactivateUpperLayer", false) ? 1 : 0;
    m.deact_uppers = in.l("Moire.TDBLDeactivateUpperLayers", false) ? 1 : 0;
    if (encapsulated) {
        const bool f2g2 = in.l("Intralayer.F2G2Model", true) && !in.l("Intralayer.RemoveF2G2Flag", false);
        const bool one = in.l("Interlayer.BilayerOneParameter", false);
        if (in.l("Intralayer.BilayerThreeParameters", false) || !(f2g2 || one))
            die("encapsulated bilayer: BilayerThreeParameters, or neither F2G2Model nor BilayerOneParameter, is not "
                "on the recursion path of this program");
        if (one) {
            m.bernal = 1;
            m.tbl[2] = -in.d("Intralayer.BilayertAB1", 0.361) / g0;
        } else {
            m.bernal = in.l("Interlayer.LegacyBernalTAB1", false) ? 1 : 2;
            static const char* keys[7] = {"Intralayer.BilayertAA1", "Intralayer.BilayertAA3", "Intralayer.BilayertAB1",
                                          "Intralayer.BilayertAB3", "Intralayer.BilayertBA0", "Intralayer.BilayertBA2",
                                          "Intralayer.BilayertBA5"};
            static const double dflt[7] = {0.09244, -0.02299, 0.1391, -0.07211, 0.331, -0.01016, 0.0001};
            for (int k = 0; k < 7; ++k) m.tbl[k] = -in.d(keys[k], dflt[k]) / g0;
        }
    }
    // moireBLShift.Calc (calc.F90:40-60, moireBLShift.F90): the rigid layer shifts tau of each calculation
    if (in.l("moireBLShift.Calc", false)) {
        if (in.l("Moire.BLShiftDefinedValues", false)) {
            j.bl_mode = 1;
            j.bl_val[0] = in.d("Moire.BilayerBottomXShift", 0.0);
            j.bl_val[1] = in.d("Moire.BilayerBottomYShift", 0.0);
            j.bl_val[2] = in.d("Moire.BilayerTopXShift", 0.0);
            j.bl_val[3] = in.d("Moire.BilayerTopYShift", 0.0);
        } else if (in.l("Moire.BLShiftRange", false)) {
            j.bl_mode = 2;
            j.bl_steps = (int)in.i("Moire.BLShiftRangeSteps", 10);
            if (j.bl_steps < 1) die("Moire.BLShiftRangeSteps must be at least 1");
            static const char* lo[4] = {"Moire.BilayerBottomXMin", "Moire.BilayerBottomYMin", "Moire.BilayerTopXMin",
                                        "Moire.BilayerTopYMin"};
            static const char* hi[4] = {"Moire.BilayerBottomXMax", "Moire.BilayerBottomYMax", "Moire.BilayerTopXMax",
                                        "Moire.BilayerTopYMax"};
            for (int k = 0; k < 4; ++k) {
                j.bl_min[k] = in.d(lo[k], 0.0);
                j.bl_max[k] = in.d(hi[k], 0.0);
            }
        }
    }
    if (bl == "Koshino" || bl == "HTC") m.interlayer = 1;
    m.vpppi0 = in.d("Interlayer.Vpppi0", koshino_intra ? 2.7 : 3.5) / g0;
    m.vppsigma0 = -in.d("Interlayer.Vppsigma0", 0.48) / g0;
    m.bl_delta = in.d("Interlayer.BLdelta", 0.184 * aG);
    m.d_interlayer = in.d("Structure.InterlayerDistance", 3.35);
    m.aCC = acc;
    m.g_intlay = in.d("TB.InterLayerHopping", 0.39) / g0;
    m.anderson = in.l("Disorder.Anderson", false) ? 1 : 0;
    m.anderson_w = in.has("Disorder.AndersonAmp") ? in.d("Disorder.AndersonAmp", 0.0) / g0 : 1.0;
    m.e0_c = in.d("TB.OnSiteC", 0.0) / g0;
    m.koshino_sr = in.l("Interlayer.KoshinoSR", false) ? 1 : 0;
    m.renormalize_coupling = in.l("Interlayer.RenormalizeCoupling", false) ? 1 : 0;
    m.coupling_factor = in.d("Interlayer.CouplingFactor", 1.0);
    j.second_layer = in.l("Interlayer.AddSecondLayerInteractions", false);
    j.nrecurs = (int)in.i("Kubo.RecursionNumber", 700);
    j.eta = in.d("Kubo.Epsilon", 0.01) / g0;
    j.n_en = (int)in.i("Kubo.NumberofEnergyPoints", 1000);
    j.emin = in.d("Kubo.EnergyMin", -4.0) / g0;
    j.emax = in.d("Kubo.EnergyMax", 4.0) / g0;
    j.seed = (int)in.i("Kubo.SeedValue", 123456);
    if (j.nrecurs < 1 || j.n_en < 1) die("Kubo.RecursionNumber and Kubo.NumberofEnergyPoints must be positive");
    // time evolution (CalcKubo, calc.F90:164-170, 545-556): it follows the DOS unless Calculate.OnlyDOS
    j.only_dos = in.l("Calculate.OnlyDOS", false);
    j.polynomials = in.l("Calculate.Polynomials", false);
    j.npol = (int)in.i("Kubo.NumberofPolynomials", 100);
    j.nt = (int)in.i("Kubo.NumberofTimeSteps", 500);
    j.nwr = (int)in.i("Kubo.WriteNumberofSteps", 10);
    j.dt = in.d("Kubo.TimeStep", 5.0);
    j.tevol_vectors = (int)in.i("Kubo.TEvolVectors", 1);   // no counterpart in the reference (one vector)
    if (j.tevol_vectors < 1 || j.tevol_vectors > 32) die("Kubo.TEvolVectors must be in 1..32");
    if (j.npol < 1 || j.nt < 0 || j.nwr < 1) die("Kubo.NumberofPolynomials and Kubo.WriteNumberofSteps must be positive");
    j.haldane = in.l("Haldane.NNN", false);
    j.hal_paper = in.l("Haldane.PaperOrientation", false);
    j.hal_opposite = in.l("Haldane.OppositePhase", false);
    j.hal_t2 = in.d("Haldane.T2", 0.0) / g0;   // HamInputEnergyEV: eV in, g0 units
    if (in.l("Haldane.SpecifyFlux", false)) {
        j.hal_mode = 1;
        j.hal_flux = in.d("Haldane.Flux", 0.0);
        j.hal_setfluxq = in.l("Haldane.SetFluxQ", false);
    } else if (in.l("Haldane.SpecifyPhase", false)) {
        j.hal_mode = 2;
        j.hal_phase = in.d("Haldane.Phase", 0.0);
    } else if (in.l("Haldane.SpecifyRange", false)) {
        j.hal_mode = 3;
        j.mphii = in.i("HaldPhase.InitialInteger", 0);
        j.mphif = in.i("HaldPhase.FinalInteger", 0);
        if (j.mphii == j.mphif && j.mphii != 0)
            die("Haldane.SpecifyRange: HaldPhase.InitialInteger = HaldPhase.FinalInteger divides the phase step by zero");
        if (j.mphii > j.mphif) die("Haldane.SpecifyRange: HaldPhase.InitialInteger is above HaldPhase.FinalInteger");
    }
    if (j.mphii != 0 || j.mphif != 0) {
        j.mphistep = in.i("HaldPhase.Step", 1);
        if (j.mphistep <= 0) j.mphistep = 1;
    }
    if (in.l("Haldane.LayerControl", false) && in.has("HaldaneLayers")) {
        for (int k = 0; k < in.count("HaldaneLayers") && k < 32; ++k) {
            const long l = in.i("HaldaneLayers", -1, k);
            if (l < 1 || l > 32) die("HaldaneLayers: layers are numbered 1..32");
            j.hal_mask |= 1u << (l - 1);
        }
        if (j.hal_mask == 0) j.hal_mask = 0x80000000u;   // a list of no layer: the term is applied nowhere
    }
    j.write_data = in.l("Output.WriteDataFiles", false);
    j.read_data = in.l("Output.ReadDataFiles", false);
    j.read_details = in.l("Neigh.ReadDetails", false);
    // local DOS selections (CalcKubo, calc.F90:214-300): the first flag that is set picks the mode
    if (in.l("Kubo.PDOS", false)) {
        gbn_pdos& p = j.pdos;
        const char* flags[10][2] = {{"Kubo.PDOSLayer", "f"}, {"Kubo.PDOSLayerAndSpecies", "f"}, {"Kubo.PDOSDist", "f"},
                                    {"Kubo.PDOSMoireSC1", "f"}, {"Kubo.PDOSMoireSuperMoire", "t"},
                                    {"Kubo.PDOSMoireSuperMoire2", "t"}, {"Kubo.PDOSMoireSuperMoire3", "t"},
                                    {"Kubo.PDOSAtomList", "f"}, {"Kubo.PDOSByNumber", "f"}, {"Kubo.PDOSPNP", "f"}};
        const int modes[10] = {GBN_PDOS_LAYER, GBN_PDOS_LAYER_SPECIES, GBN_PDOS_DIST, GBN_PDOS_MOIRE_SC1,
                               GBN_PDOS_SUPERMOIRE, GBN_PDOS_SUPERMOIRE2, GBN_PDOS_SUPERMOIRE3, GBN_PDOS_ATOM_LIST,
                               GBN_PDOS_BY_NUMBER, GBN_PDOS_PNP};
        for (int k = 0; k < 10 && p.mode == 0; ++k)
            if (in.l(flags[k][0], flags[k][1][0] == 't')) p.mode = modes[k];
        p.xmin = in.d("Kubo.PDOSxmin", 0.0);
        p.xmax = in.d("Kubo.PDOSxmax", 5.0);
        p.ymin = in.d("Kubo.PDOSymin", 0.0);
        p.ymax = in.d("Kubo.PDOSymax", 5.0);
        p.min_value = (int32_t)in.i("Kubo.PDOSMinValue", 0);
        p.super_cell = j.cell.super_cell;
        p.cell_size = j.cell.cell_size;
        p.supermoire_length = in.d("Kubo.PDOSMoireSuperMoireLength", 135.0);
        p.aG = aG;
        p.ignore_layers_1_4 = in.l("Kubo.PDOSIgnoreLayer1and4", false) ? 1 : 0;
        for (int k = 0; k < 6; ++k) p.atom_list[k] = (int32_t)(in.has("Kubo.PDOSList") ? in.i("Kubo.PDOSList", 0, k) : k + 1);
        p.atom_number = (int32_t)in.i("Kubo.PDOSNumber", 1);
        p.pnp_delta = in.d("Potential.PNPDelta", 10.0);
        p.number_of_layers = (int32_t)in.i("Kubo.NumberOfLayers", 2);
        p.n_bn1 = (int32_t)in.i("Kubo.NumberOfBNAtoms1", 5832);
        p.n_bn2 = (int32_t)in.i("Kubo.NumberOfBNAtoms2", 5832);
        p.n_c = (int32_t)in.i("Kubo.NumberOfCAtoms", 6050);
        p.stack = in.l("Stack.EncapsulatedFourLayers", false) ? GBN_STACK_ENCAPSULATED_FOUR
                                                              : (in.l("Stack.T3BG", false) ? GBN_STACK_T3BG : GBN_STACK_NONE);
        j.seed_set = (int)in.i("Kubo.SeedSet", 1235);
    }
    // field sweep (MagfInit, magf.F90:20-98); values in tesla are converted once the cell area is known
    if (in.has("MagField.Value")) {
        j.field_by_value = true;
        j.b_value = in.d("MagField.Value", 0.0);
    } else if (in.has("MagField.Integer")) {
        j.mbi = j.mbf = in.i("MagField.Integer", 0);
    } else if (in.has("MagField.InitialB")) {
        j.field_steps_by_value = true;
        j.b_init = in.d("MagField.InitialB", 0.0);
        j.b_final = in.d("MagField.FinalB", 0.0);
    } else if (in.has("MagField.InitialInteger")) {
        j.mbi = in.i("MagField.InitialInteger", 0);
        j.mbf = in.i("MagField.FinalInteger", 0);
        if (j.mbi > j.mbf) die("MagField.InitialInteger is above MagField.FinalInteger");
    }
    j.b_step = in.has("MagField.Step") ? in.d("MagField.Step", 1.0) : 0.0;
    j.mstep = in.i("MagField.IntegerStep", 1);
    j.prefix = in.s("Run.Prefix", "grabnes");
    return j;
}

double cell_area(const double* u)
{
    const double v1 = u[1] * u[5] - u[2] * u[4], v2 = u[2] * u[3] - u[0] * u[5], v3 = u[0] * u[4] - u[1] * u[3];
    return sqrt(v1 * v1 + v2 * v2 + v3 * v3);
}

// field sweep in flux quanta through the cell, once the area is known
void resolve_fields(Job& j, double area)
{
    auto quanta = [&](double bmag) { return lround(area * 1.0e-20 * bmag / kFluxQuantum); };
    if (j.field_by_value) j.mbi = j.mbf = quanta(j.b_value);
    if (j.field_steps_by_value) {
        j.mbi = quanta(j.b_init);
        j.mbf = quanta(j.b_final);
        if (j.mbi > j.mbf) die("MagField.InitialB is above MagField.FinalB");
    }
    if (j.b_step > 0.0) j.mstep = quanta(j.b_step);
    if (j.mstep <= 0) j.mstep = 1;
}

// a double as gfortran's list-directed output writes it: 17 significant digits in a 25-wide field, fixed
// notation for 0.1 <= |x| < 1e16, otherwise a mantissa and a three-digit exponent.  The decimal exponent
// is taken from the correctly rounded 17-digit form, so the text always reads back to the same double.
std::string fortran_ld(double x)
{
    char sci[64], buf[80];
    snprintf(sci, sizeof sci, "%.16e", x);
    const char* ep = strchr(sci, 'e');
    const int e = ep ? atoi(ep + 1) : 0;
    if (!std::isfinite(x)) {   // gfortran's list-directed NaN / Infinity
        snprintf(buf, sizeof buf, "%26s", std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
    } else if (x == 0.0) {
        snprintf(buf, sizeof buf, "   0.0000000000000000     ");
    } else if (e >= -1 && e < 16) {
        snprintf(buf, sizeof buf, "   %.*f     ", 16 - e, x);
    } else {
        const std::string mant(sci, ep ? (size_t)(ep - sci) : strlen(sci));
        snprintf(buf, sizeof buf, "   %sE%c%03d", mant.c_str(), e < 0 ? '-' : '+', abs(e));
    }
    return buf;
}

void write_column(const std::string& path, const std::vector<double>& v)
{
    FILE* f = fopen(path.c_str(), "w");
    if (!f) die("cannot write " + path);
    for (double x : v) fprintf(f, "%s\n", fortran_ld(x).c_str());
    fclose(f);
}

void ck(int rc, gbn_ctx* ctx, const char* what)
{
    if (rc != GBN_OK) die(std::string(what) + ": " + (ctx ? gbn_last_error(ctx) : "error " + std::to_string(rc)));
}

// Sweep sharding over processes, one per GPU (grabnes_b200/launch.py starts them): GRABNES_RANK and
// GRABNES_NRANKS.  Unit u of a sweep -- the u-th (field, Haldane phase) pair in the reference's loop
// order (calc.F90:82-114), or the u-th field of a batched DOS-only sweep, the same order -- runs on rank
// u % NRANKS and writes its own folder; a job without a sweep is one unit.  No data crosses ranks.
struct Shard {
    int rank = 0, nranks = 1;
    bool mine(long u) const { return u % nranks == rank; }
};

Shard shard_from_env()
{
    Shard s;
    const char* r = getenv("GRABNES_RANK");
    const char* n = getenv("GRABNES_NRANKS");
    if (n) s.nranks = atoi(n);
    if (r) s.rank = atoi(r);
    if (s.nranks < 1 || s.rank < 0 || s.rank >= s.nranks) die("GRABNES_RANK must be in 0 .. GRABNES_NRANKS - 1");
    return s;
}

// moireBLShiftValue (moireBLShift.F90:57-110): the layer shifts (tauX1, tauY1, tauX2, tauY2) of each
// calculation of a moireBLShift.Calc sweep, tau = min + mS (max - min) / steps for mS = 0 .. steps, and for a
// range its folder X1_<tauX1>_Y1_<tauY1>_X2_<tauX2>_Y2_<tauY2> (the f0.4 values).  Without a range: one
// calculation, with the defined values or 0, in the run's own prefix.
struct ShiftUnit {
    double tau[4] = {0, 0, 0, 0};
    std::string folder;
};

std::vector<ShiftUnit> shift_units(const Job& j)
{
    std::vector<ShiftUnit> out;
    if (j.bl_mode == 2) {
        for (int mS = 0; mS <= j.bl_steps; ++mS) {
            ShiftUnit u;
            for (int k = 0; k < 4; ++k)
                u.tau[k] = j.bl_min[k] + (double)mS * (j.bl_max[k] - j.bl_min[k]) / (double)j.bl_steps;
            char f[192];
            snprintf(f, sizeof f, "X1_%.4f_Y1_%.4f_X2_%.4f_Y2_%.4f", u.tau[0], u.tau[1], u.tau[2], u.tau[3]);
            u.folder = f;
            out.push_back(u);
        }
    } else {
        ShiftUnit u;
        if (j.bl_mode == 1)
            for (int k = 0; k < 4; ++k) u.tau[k] = j.bl_val[k];
        out.push_back(u);
    }
    return out;
}

// The (field, phase) units of the sweep in loop order (integer fields, before MagField.*B is resolved); for
// a layer-shift range, its shifts (mS, 0).
std::vector<std::pair<long, long>> sweep_units(const Job& j)
{
    std::vector<std::pair<long, long>> u;
    if (j.bl_mode == 2) {
        for (long mS = 0; mS <= j.bl_steps; ++mS) u.push_back({mS, 0});
        return u;
    }
    const bool magfield = !(j.mbi == 0 && j.mbf == 0), hsweep = j.mphii != j.mphif;
    for (long mb = j.mbi; mb <= j.mbf; mb += (magfield ? j.mstep : 1)) {
        for (long mphi = j.mphii; mphi <= j.mphif; mphi += j.mphistep) {
            u.push_back({mb, mphi});
            if (!magfield && !hsweep) return u;
        }
    }
    return u;
}

void print_job(const Job& j)
{
    {   // the units of this rank (GRABNES_RANK / GRABNES_NRANKS), on a line of their own before the job
        const Shard sh = shard_from_env();
        const auto units = sweep_units(j);
        printf("{\"rank\": %d, \"nranks\": %d, \"units\": [", sh.rank, sh.nranks);
        bool first = true;
        for (size_t k = 0; k < units.size(); ++k)
            if (sh.mine((long)k)) {
                printf("%s[%ld, %ld]", first ? "" : ", ", units[k].first, units[k].second);
                first = false;
            }
        printf("]}\n");
    }
    const gbn_model& m = j.model;
    printf("{\"kind\": %d, \"aG\": %.17g, \"cell_size\": %d, \"super_cell\": %d, \"m\": [%d, %d, %d, %d], "
           "\"height\": %.17g, \"d_interlayer\": %.17g, \"g0\": %.17g, \"cut2intra\": %.17g, \"cut2inter\": %.17g, "
           "\"second_layer\": %d, \"moire\": %d, \"nrecurs\": %d, \"eta\": %.17g, \"n_en\": %d, \"emin\": %.17g, "
           "\"emax\": %.17g, \"seed\": %d, \"prefix\": \"%s\", \"only_dos\": %d, \"npol\": %d, \"nt\": %d, "
           "\"nwr\": %d, \"dt\": %.17g, \"pdos_mode\": %d, \"seed_set\": %d, \"haldane\": %d, \"hal_t2\": %.17g, "
           "\"hal_mode\": %d, \"mphi\": [%ld, %ld, %ld], \"model\": {\"tbnn\": %d, \"intralayer\": %d, "
           "\"moire_onsite\": %d, \"moire_offdiag\": %d, \"moire_mid\": %d, \"moire_twisted\": %d, \"eps\": %.17g, "
           "\"twist_rad\": %.17g, \"C0\": %.17g, \"Cz\": %.17g, \"Cab\": %.17g, \"interlayer\": %d, "
           "\"vpppi0\": %.17g, \"vppsigma0\": %.17g, \"bl_delta\": %.17g, \"anderson\": %d, \"anderson_w\": %.17g, "
           "\"tksl2\": %.17g, \"koshino_sr\": %d, \"renormalize_coupling\": %d, \"coupling_factor\": %.17g, "
           "\"second_moire\": %d, \"eps_factor\": %.17g, \"twisted2\": %d, \"twist2_rad\": %.17g, "
           "\"rotate_first\": %d, \"shift2_x\": %.17g, \"shift2_y\": %.17g, \"sign2\": %.17g, "
           "\"encapsulated\": %d, \"bl_bottom_rad\": %.17g, \"bl_top_rad\": %.17g, \"deact_upper\": %d, "
           "\"deact_uppers\": %d, \"bernal\": %d, \"tbl\": [%.17g, %.17g, %.17g, %.17g, %.17g, %.17g, %.17g]}, "
           "\"add_shift\": %d, \"shift_factor\": %.17g, \"bl_mode\": %d, \"bl_steps\": %d}\n",
           j.cell.kind, j.cell.aG, j.cell.cell_size, j.cell.super_cell, j.cell.m[0], j.cell.m[1], j.cell.m[2], j.cell.m[3],
           j.cell.height, j.cell.d_interlayer, j.g0, j.cut2intra, j.cut2inter, (int)j.second_layer, (int)j.moire,
           j.nrecurs, j.eta, j.n_en, j.emin, j.emax, j.seed, j.prefix.c_str(), (int)j.only_dos, j.npol, j.nt, j.nwr,
           j.dt, j.pdos.mode, j.seed_set, (int)j.haldane, j.hal_t2, j.hal_mode, j.mphii, j.mphif, j.mphistep, m.tbnn, m.intralayer, m.moire_onsite,
           m.moire_offdiag, m.moire_mid, m.moire_twisted, m.eps, m.twist_rad, m.C0, m.Cz, m.Cab, m.interlayer,
           m.vpppi0, m.vppsigma0, m.bl_delta, m.anderson, m.anderson_w, m.tksl[2], m.koshino_sr,
           m.renormalize_coupling, m.coupling_factor, m.second_moire, m.eps_factor, m.twisted2, m.twist2_rad,
           m.rotate_first, m.shift2_x, m.shift2_y, m.sign2, m.encapsulated, m.bl_bottom_rad, m.bl_top_rad,
           m.deact_upper, m.deact_uppers, m.bernal, m.tbl[0], m.tbl[1], m.tbl[2], m.tbl[3], m.tbl[4], m.tbl[5],
           m.tbl[6], j.cell.add_shift, j.cell.shift_factor, j.bl_mode, j.bl_steps);
}

void write_pairs(const std::string& path, const std::vector<double>& x, const std::vector<double>& y, double head,
                 bool with_head)
{
    FILE* f = fopen(path.c_str(), "w");
    if (!f) die("cannot write " + path);
    if (with_head) fprintf(f, "%s\n", fortran_ld(head).c_str());
    for (size_t k = 0; k < x.size(); ++k) fprintf(f, "%s%s\n", fortran_ld(x[k]).c_str(), fortran_ld(y[k]).c_str());
    fclose(f);
}

// KuboInterval + KuboCn (<prefix>.cn.dat: Re c_n and |c_n|), then, without Calculate.OnlyDOS, KuboTEvol
// (kubo.F90:321-397): nT steps of KuboEvol along x from the start vector psi with zupsi = 0; every nWr
// steps the recursion of zupsi / |zupsi| and the continued fraction weighted by |zupsi|^2 are written
// to <prefix>.Z2_<step>.dat and <prefix>.AB_<step>.dat.
void time_evolution(gbn_ctx* ctx, const Job& j, std::vector<double> psi, const std::vector<double>& a,
                    const std::vector<double>& b, const std::string& prefix, int64_t n)
{
    double ac = 0.0, bc = 0.0;
    ck(gbn_cheb_interval(a.data(), b.data(), j.nrecurs, &ac, &bc), nullptr, "gbn_cheb_interval");
    std::vector<double> c((size_t)2 * j.npol);
    ck(gbn_cheb_coef(j.dt, ac, bc, j.npol, c.data()), nullptr, "gbn_cheb_coef");
    std::vector<double> re((size_t)j.npol), ab((size_t)j.npol);
    for (int k = 0; k < j.npol; ++k) {
        re[(size_t)k] = c[(size_t)2 * k];
        ab[(size_t)k] = hypot(c[(size_t)2 * k], c[(size_t)2 * k + 1]);
    }
    write_pairs(prefix + ".cn.dat", re, ab, 0.0, false);
    if (j.only_dos) return;
    // all nT steps on the device (gbn_kubo_tevol); the files of every nWr-th step from its coefficients.
    // Vector 0 is the reference's start vector; Kubo.TEvolVectors > 1 adds random-phase vectors from the
    // continuation of the same seeded stream (vector r: draws r N .. (r + 1) N - 1), batched in one call.
    const int R = j.tevol_vectors;
    if ((int64_t)psi.size() != 2 * n) die("time evolution without a start vector");
    psi.resize((size_t)2 * n * R);
    if (R > 1) {
        std::vector<double> u((size_t)n * R);
        ck(gbn_rng_uniform(j.seed, n * R, u.data()), nullptr, "gbn_rng_uniform");
        const double isn = 1.0 / sqrt((double)n);
        for (int r = 1; r < R; ++r)
            for (int64_t i = 0; i < n; ++i) {
                const double ph = 2.0 * kPi * u[(size_t)r * n + i];
                psi[(size_t)2 * ((size_t)r * n + i)] = cos(ph) * isn;
                psi[(size_t)2 * ((size_t)r * n + i) + 1] = sin(ph) * isn;
            }
    }
    std::vector<double> zu((size_t)2 * n * R, 0.0);
    const int nw = j.nt / j.nwr;
    const int nw1 = std::max(nw, 1);
    std::vector<double> norms((size_t)R * nw1), az((size_t)R * nw1 * j.nrecurs), bz((size_t)R * nw1 * j.nrecurs),
        energy((size_t)j.n_en + 1), dos((size_t)j.n_en + 1);
    ck(gbn_kubo_tevol(ctx, GBN_FP64, R, c.data(), j.npol, ac, bc, 1, j.nt, j.nwr, j.nrecurs, psi.data(), zu.data(),
                      norms.data(), az.data(), bz.data()),
       ctx, "gbn_kubo_tevol");
    if (nw > 0) {   // <prefix>.MSD.dat: spread and diffusivity, the mean over the vectors
        std::vector<double> nr((size_t)R * nw), t((size_t)nw), msd((size_t)nw), dr((size_t)nw), ds((size_t)nw);
        for (int r = 0; r < R; ++r)
            for (int w = 0; w < nw; ++w) nr[(size_t)r * nw + w] = norms[(size_t)r * nw1 + w];
        const double dt_fs = j.dt * (kHPLANCK / (2.0 * kPi)) / kQE / j.g0 * 1e15;
        ck(gbn_kubo_msd(R, nw, j.nwr, dt_fs, nr.data(), t.data(), msd.data(), dr.data(), ds.data()), nullptr,
           "gbn_kubo_msd");
        FILE* f = fopen((prefix + ".MSD.dat").c_str(), "w");
        if (!f) die("cannot write " + prefix + ".MSD.dat");
        fprintf(f, "# %d vector(s), direction x: t [fs], MSD = <(X(t) - X(0))^2> [Ang^2], MSD / t [Ang^2/fs], "
                   "d MSD / dt [Ang^2/fs]\n", R);
        for (int w = 0; w < nw; ++w)
            fprintf(f, "%.16e %.16e %.16e %.16e\n", t[(size_t)w], msd[(size_t)w], dr[(size_t)w], ds[(size_t)w]);
        fclose(f);
    }
    for (int w = 0; w < nw; ++w) {
        const int it = (w + 1) * j.nwr;
        double norm = norms[(size_t)w];
        if (!(norm > 0.0)) continue;
        std::vector<double> aw(az.begin() + (size_t)w * j.nrecurs, az.begin() + (size_t)(w + 1) * j.nrecurs);
        std::vector<double> bw(bz.begin() + (size_t)w * j.nrecurs, bz.begin() + (size_t)(w + 1) * j.nrecurs);
        ck(gbn_cf_dos(ctx, 1, aw.data(), bw.data(), nullptr, j.nrecurs, j.eta, j.n_en, j.emin, j.emax, &norm,
                      energy.data(), dos.data()),
           ctx, "gbn_cf_dos");
        char tag[32];
        snprintf(tag, sizeof tag, "%04d", it);
        write_pairs(prefix + ".Z2_" + tag + ".dat", energy, dos, 0.0, false);
        write_pairs(prefix + ".AB_" + tag + ".dat", aw, bw, norm, true);
        printf("grabnes: time step %d of %d, |ZUPsi|^2 = %.10g\n", it, j.nt, norm);
    }
}

// A list-directed real of gfortran without its padding (for complex pairs).
std::string ld_trim(double x)
{
    std::string t = fortran_ld(x);
    const size_t a = t.find_first_not_of(' '), b = t.find_last_not_of(' ');
    return a == std::string::npos ? t : t.substr(a, b - a + 1);
}

FILE* open_or_die(const std::string& path)
{
    FILE* f = fopen(path.c_str(), "w");
    if (!f) die("cannot write " + path);
    return f;
}

// Output.WriteDataFiles, neighbour part (NeighWriteDataFiles, neigh.F90:383-440): v, dx, dy, dz, pos,
// neighCell.dat, neighD.dat in the working folder, with the reference's edit descriptors.
void write_neigh_files(gbn_ctx* ctx, int64_t n, int32_t maxn, const std::vector<double>& rat,
                       const std::vector<int32_t>& species)
{
    std::vector<int32_t> nn((size_t)n), nl((size_t)n * maxn), nc((size_t)3 * n * maxn);
    std::vector<double> nd((size_t)3 * n * maxn);
    ck(gbn_get_neighbours(ctx, nn.data(), nl.data(), nd.data(), nc.data()), ctx, "gbn_get_neighbours");
    FILE* fv = open_or_die("v");
    FILE* fx[3] = {open_or_die("dx"), open_or_die("dy"), open_or_die("dz")};
    FILE* fp = open_or_die("pos");
    FILE* fc = open_or_die("neighCell.dat");
    FILE* fd = open_or_die("neighD.dat");
    for (int64_t i = 0; i < n; ++i) {
        const int k = nn[(size_t)i];
        const size_t e0 = (size_t)i * maxn;
        fprintf(fv, "%12d\n", k);
        for (int j = 0; j < k; ++j) fprintf(fv, "%8d %s", nl[e0 + j], (j % 500 == 499 && j + 1 < k) ? "\n" : "");
        fprintf(fv, "\n");
        for (int c = 0; c < 3; ++c) {
            for (int j = 0; j < k; ++j)
                fprintf(fx[c], "%10.5f %s", nd[3 * (e0 + j) + c], (j % 500 == 499 && j + 1 < k) ? "\n" : "");
            fprintf(fx[c], "\n");
        }
        const char* label = species[(size_t)i] == 3 ? "B    " : (species[(size_t)i] == 4 ? "N    " : "C    ");
        fprintf(fp, " %s%s%s%s\n", label, fortran_ld(rat[(size_t)3 * i]).c_str(), fortran_ld(rat[(size_t)3 * i + 1]).c_str(),
                fortran_ld(rat[(size_t)3 * i + 2]).c_str());
        for (int j = 0; j < k; ++j) {
            const size_t e = e0 + j;
            fprintf(fc, "%6d %6d %6d \n", nc[3 * e], nc[3 * e + 1], nc[3 * e + 2]);
            fprintf(fd, "%24.16E %24.16E %24.16E \n", nd[3 * e], nd[3 * e + 1], nd[3 * e + 2]);
        }
    }
    for (FILE* f : {fv, fx[0], fx[1], fx[2], fp, fc, fd}) fclose(f);
    printf("grabnes: neighbour tables written (v, dx, dy, dz, pos, neighCell.dat, neighD.dat)\n");
}

// Output.WriteDataFiles, Hamiltonian part (HamHopping and HamHopWriteTables, ham.F90:6944-7040):
// <prefix>.s.mag (the hoppings of each atom, g0 units, the reference's sign), <prefix>.e (H0, Species,
// layerIndex), <prefix>.pos, <prefix>.cell (ucell then the reciprocal cell, one vector per line), and the
// empty <prefix>.HABreal / .HABimag of models without those terms, <prefix>.bottom.e and (second moire)
// <prefix>.top.e.
void write_ham_files(gbn_ctx* ctx, const std::string& prefix, int64_t n, int32_t maxn, const std::vector<double>& rat,
                     const std::vector<int32_t>& species, const std::vector<int32_t>& layer, const double* u,
                     bool second_moire)
{
    std::vector<int32_t> nn((size_t)n);
    ck(gbn_get_neighbours(ctx, nn.data(), nullptr, nullptr, nullptr), ctx, "gbn_get_neighbours");
    std::vector<double> h0((size_t)n), hop((size_t)2 * n * maxn);
    ck(gbn_get_hamiltonian(ctx, h0.data(), hop.data()), ctx, "gbn_get_hamiltonian");
    FILE* f = open_or_die(prefix + ".s.mag");
    for (int64_t i = 0; i < n; ++i) {
        for (int j = 0; j < nn[(size_t)i]; ++j) {
            const size_t e = (size_t)i * maxn + j;
            fprintf(f, " (%s,%s)", ld_trim(hop[2 * e]).c_str(), ld_trim(hop[2 * e + 1]).c_str());
        }
        fprintf(f, "\n");
    }
    fclose(f);
    f = open_or_die(prefix + ".e");
    for (int64_t i = 0; i < n; ++i)
        fprintf(f, "%s%12d%12d\n", fortran_ld(h0[(size_t)i]).c_str(), species[(size_t)i], layer[(size_t)i]);
    fclose(f);
    fclose(open_or_die(prefix + ".HABreal"));
    fclose(open_or_die(prefix + ".HABimag"));
    f = open_or_die(prefix + ".pos");
    for (int64_t i = 0; i < n; ++i)
        fprintf(f, "%s%s%s\n", fortran_ld(rat[(size_t)3 * i]).c_str(), fortran_ld(rat[(size_t)3 * i + 1]).c_str(),
                fortran_ld(rat[(size_t)3 * i + 2]).c_str());
    fclose(f);
    // rcell(:,k) = 2 pi (ucell(:,k+1) x ucell(:,k+2)) / volume (cell.F90:400-402)
    auto cross = [](const double* x, const double* y, double* z) {
        z[0] = x[1] * y[2] - x[2] * y[1];
        z[1] = x[2] * y[0] - x[0] * y[2];
        z[2] = x[0] * y[1] - x[1] * y[0];
    };
    double c12[3];
    cross(u, u + 3, c12);
    const double vol = fabs(c12[0] * u[6] + c12[1] * u[7] + c12[2] * u[8]);
    double rc[9];
    cross(u + 3, u + 6, rc);
    cross(u + 6, u, rc + 3);
    cross(u, u + 3, rc + 6);
    f = open_or_die(prefix + ".cell");
    for (int v = 0; v < 3; ++v)
        fprintf(f, "%s%s%s\n", fortran_ld(u[3 * v]).c_str(), fortran_ld(u[3 * v + 1]).c_str(), fortran_ld(u[3 * v + 2]).c_str());
    for (int v = 0; v < 3; ++v)
        fprintf(f, "%s%s%s\n", fortran_ld(2.0 * kPi * rc[3 * v] / vol).c_str(), fortran_ld(2.0 * kPi * rc[3 * v + 1] / vol).c_str(),
                fortran_ld(2.0 * kPi * rc[3 * v + 2] / vol).c_str());
    fclose(f);
    // <prefix>.bottom.e (always) and <prefix>.top.e (Moire.AddSecondMoire): H0Bottom / H0Top and Species,
    // ham.F90:7020-7034
    std::vector<double> bottom((size_t)n), top((size_t)n);
    ck(gbn_get_onsite_layers(ctx, bottom.data(), top.data()), ctx, "gbn_get_onsite_layers");
    f = open_or_die(prefix + ".bottom.e");
    for (int64_t i = 0; i < n; ++i) fprintf(f, "%s%12d\n", fortran_ld(bottom[(size_t)i]).c_str(), species[(size_t)i]);
    fclose(f);
    if (second_moire) {
        f = open_or_die(prefix + ".top.e");
        for (int64_t i = 0; i < n; ++i) fprintf(f, "%s%12d\n", fortran_ld(top[(size_t)i]).c_str(), species[(size_t)i]);
        fclose(f);
    }
}

// Output.ReadDataFiles: the neighbour list from v (NeighReadDataFiles, neigh.F90:446-522: with
// Neigh.ReadDetails also neighCell.dat and neighD.dat, otherwise each entry's image is the one of the nine
// in-plane images closer than aG/sqrt(3)*1.1, the last found), H0 from generate.e and the hoppings from
// generate.s, one 're im' pair per entry (calc.F90:86-95, ham.F90:659-672).
struct Tables {
    int32_t maxn = 0;
    std::vector<int32_t> nn, nl, nc;
    std::vector<double> nd, h0, hop;
};

std::vector<double> read_numbers(const std::string& path, bool first_column_only)
{
    FILE* f = fopen(path.c_str(), "r");
    if (!f) die("Output.ReadDataFiles: cannot open " + path);
    std::vector<double> out;
    char line[1 << 16];
    while (fgets(line, sizeof line, f)) {
        for (char* q = line; *q; ++q)
            if (*q == 'd' || *q == 'D') *q = 'e';   // Fortran double-precision exponents
        char* p = line;
        for (;;) {
            char* end = nullptr;
            const double v = strtod(p, &end);
            if (end == p) break;
            out.push_back(v);
            p = end;
            if (first_column_only) break;
        }
    }
    fclose(f);
    return out;
}

Tables read_tables(const Job& j, int64_t n, const std::vector<double>& ucell, const std::vector<double>& rat)
{
    Tables t;
    const std::vector<double> v = read_numbers("v", false);
    t.nn.assign((size_t)n, 0);
    std::vector<std::vector<int32_t>> rows((size_t)n);
    size_t p = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (p >= v.size()) die("Output.ReadDataFiles: v ends before atom " + std::to_string(i + 1));
        const int k = (int)v[p++];
        if (k < 0 || p + (size_t)k > v.size()) die("Output.ReadDataFiles: v is inconsistent at atom " + std::to_string(i + 1));
        t.nn[(size_t)i] = k;
        for (int q = 0; q < k; ++q) rows[(size_t)i].push_back((int32_t)v[p++]);
        t.maxn = std::max(t.maxn, k);
    }
    t.maxn = std::max(t.maxn, 1);
    const size_t E = (size_t)n * t.maxn;
    t.nl.assign(E, 1);
    t.nc.assign(3 * E, 0);
    t.nd.assign(3 * E, 0.0);
    for (int64_t i = 0; i < n; ++i)
        for (int q = 0; q < t.nn[(size_t)i]; ++q) {
            const int32_t m = rows[(size_t)i][(size_t)q];
            if (m < 1 || m > n) die("Output.ReadDataFiles: neighbour index outside 1..N in v");
            t.nl[(size_t)i * t.maxn + q] = m;
        }
    if (j.read_details) {
        const std::vector<double> c = read_numbers("neighCell.dat", false), d = read_numbers("neighD.dat", false);
        size_t q3 = 0;
        for (int64_t i = 0; i < n; ++i)
            for (int q = 0; q < t.nn[(size_t)i]; ++q, q3 += 3) {
                if (q3 + 3 > c.size() || q3 + 3 > d.size()) die("Output.ReadDataFiles: neighCell.dat / neighD.dat too short");
                for (int k = 0; k < 3; ++k) {
                    t.nc[3 * ((size_t)i * t.maxn + q) + k] = (int32_t)c[q3 + k];
                    t.nd[3 * ((size_t)i * t.maxn + q) + k] = d[q3 + k];
                }
            }
    } else {
        const double cut = j.cell.aG / sqrt(3.0) * 1.1;
        for (int64_t i = 0; i < n; ++i)
            for (int q = 0; q < t.nn[(size_t)i]; ++q) {
                const int64_t m = t.nl[(size_t)i * t.maxn + q] - 1;
                for (int ix = -1; ix <= 1; ++ix)
                    for (int iy = -1; iy <= 1; ++iy) {
                        if (i == m && ix == 0 && iy == 0) continue;
                        double w[3], d2 = 0.0;
                        for (int k = 0; k < 3; ++k) {
                            w[k] = rat[(size_t)3 * i + k] - rat[(size_t)3 * m + k] - (ix * ucell[k] + iy * ucell[3 + k]);
                            d2 += w[k] * w[k];
                        }
                        if (sqrt(d2) < cut) {
                            const size_t e = (size_t)i * t.maxn + q;
                            t.nc[3 * e] = ix; t.nc[3 * e + 1] = iy; t.nc[3 * e + 2] = 0;
                            for (int k = 0; k < 3; ++k) t.nd[3 * e + k] = -w[k];
                        }
                    }
            }
    }
    t.h0 = read_numbers("generate.e", true);
    if ((int64_t)t.h0.size() < n) die("Output.ReadDataFiles: generate.e has fewer lines than atoms");
    t.h0.resize((size_t)n);
    const std::vector<double> s = read_numbers("generate.s", false);
    t.hop.assign(2 * E, 0.0);
    size_t q2 = 0;
    for (int64_t i = 0; i < n; ++i)
        for (int q = 0; q < t.nn[(size_t)i]; ++q, q2 += 2) {
            if (q2 + 2 > s.size()) die("Output.ReadDataFiles: generate.s has fewer entries than the neighbour list");
            t.hop[2 * ((size_t)i * t.maxn + q)] = s[q2];
            t.hop[2 * ((size_t)i * t.maxn + q) + 1] = s[q2 + 1];
        }
    printf("grabnes: neighbour list, on-site energies and hoppings read from v, generate.e, generate.s\n");
    return t;
}

// The end of HamHopping (ham.F90:6940-6941): HamCheckFinite stops on non-finite values; HamCheckHermiticity
// reports the largest asymmetry of the two directions of a bond for the models with position-dependent
// bond terms (here Moire.OffDiag, and Haldane.NNN with Haldane.SpecifyPhase).
void check_hamiltonian(gbn_ctx* ctx, const Job& j)
{
    int64_t cnt[5] = {0, 0, 0, 0, 0};
    double asym = 0.0;
    ck(gbn_check_hamiltonian(ctx, cnt, &asym), ctx, "gbn_check_hamiltonian");
    if (cnt[0] + cnt[1] > 0)
        die("The Hamiltonian contains non-finite values: " + std::to_string(cnt[0]) + " hopping and " +
            std::to_string(cnt[1]) + " on-site entries (first at atom " + std::to_string(cnt[2]) + ")");
    const bool od = j.model.moire_offdiag != 0, hphase = j.haldane && j.hal_mode == 2;
    if (!(od || hphase)) return;
    if (cnt[3] > 0) printf("grabnes: hopping table: %lld entries without reverse entry\n", (long long)cnt[3]);
    const double ev = asym * j.g0;
    if (hphase && !od) {
        if (ev > 1.0e-9)
            printf("grabnes: warning: the hopping table is NOT Hermitian with HaldaneNNN and HaldaneSpecifyPhase: the "
                   "two directions of a bond differ by up to %.6g eV\n", ev);
    } else if (od && j.model.moire_mid) {
        printf("grabnes: hopping table with MoireOffDiagMidpoint: the two directions of a bond differ by up to %.6g eV\n",
               ev);
    } else {
        printf("grabnes: warning: the hopping table is NOT Hermitian: the two directions of a bond differ by up to "
               "%.6g eV, because MoireOffDiag is evaluated at the first atom of each bond. Set MoireOffDiagMidpoint "
               ".true. to evaluate it at the bond midpoint (Hermitian).\n", ev);
    }
}

// KuboDOS (kubo.F90:276-319) after the recursion: <prefix>.b0.dat, .a0.dat (KuboRecursion's files), the
// continued fraction <prefix>.DOS and the coefficients <prefix>.AB.
void kubo_dos_files(gbn_ctx* ctx, const Job& j, const std::string& prefix, const double* a, const double* b)
{
    std::vector<double> av(a, a + j.nrecurs), bv(b, b + j.nrecurs), energy((size_t)j.n_en + 1), dos((size_t)j.n_en + 1);
    write_column(prefix + ".b0.dat", bv);
    write_column(prefix + ".a0.dat", av);
    ck(gbn_cf_dos(ctx, 1, a, b, nullptr, j.nrecurs, j.eta, j.n_en, j.emin, j.emax, nullptr, energy.data(), dos.data()),
       ctx, "gbn_cf_dos");
    write_pairs(prefix + ".DOS", energy, dos, 0.0, false);
    write_pairs(prefix + ".AB", av, bv, 1.0, true);
    printf("grabnes: DOS written to %s.DOS and %s.AB\n", prefix.c_str(), prefix.c_str());
}

std::string make_folder(const std::string& name, const std::string& sysname)
{
    if (mkdir(name.c_str(), 0755) != 0 && errno != EEXIST) die("cannot create folder " + name);
    printf("grabnes: writing files in folder '%s'\n", name.c_str());
    return "./" + name + "/" + sysname;
}

// One Kubo.PDOS pass (CalcKubo, calc.F90:300-541).  All start vectors of the selection run as one batch
// of right-hand sides; the files of each go to its PDOS_* folder as the reference writes them.  On return
// psi, a, b and prefix are those of the last start vector, which the time evolution continues from.
void pdos_pass(gbn_ctx* ctx, const Job& j, int64_t n, const std::vector<double>& rat_now,
               const std::vector<int32_t>& species, const std::vector<int32_t>& layer, const std::vector<double>& ucell,
               std::vector<double>& psi, std::vector<double>& a, std::vector<double>& b, std::string& prefix, bool& any)
{
    const gbn_pdos& p = j.pdos;
    any = false;
    if (p.mode == GBN_PDOS_LAYER || p.mode == GBN_PDOS_LAYER_SPECIES) {
        int32_t maxl = 0;
        for (int32_t l : layer) maxl = l > maxl ? l : maxl;
        if (p.mode == GBN_PDOS_LAYER && p.number_of_layers < maxl)
            printf("grabnes: warning: Kubo.NumberOfLayers is %d but the structure has %d layers: the layer DOS of "
                   "layers above %d is not written\n", p.number_of_layers, maxl, p.number_of_layers);
        const int32_t cap = 4096;
        std::vector<int32_t> set_of_atom((size_t)n), sl(cap), ss(cap);
        std::vector<double> assumed(cap);
        int32_t ns = 0;
        ck(gbn_pdos_sets(&p, n, species.data(), layer.data(), cap, &ns, set_of_atom.data(), sl.data(), ss.data(),
                         assumed.data()),
           nullptr, "gbn_pdos_sets");
        if (ns == 0) return;
        std::vector<double> u((size_t)n);
        ck(gbn_rng_uniform(j.seed_set, n, u.data()), nullptr, "gbn_rng_uniform");
        std::vector<int64_t> count((size_t)ns, 0);
        for (int64_t i = 0; i < n; ++i)
            if (set_of_atom[(size_t)i] >= 0) ++count[(size_t)set_of_atom[(size_t)i]];
        for (int s = 0; s < ns; ++s)
            if (count[(size_t)s] == 0)
                printf("grabnes: warning: layer %d has no atoms: its DOS is undefined\n", sl[(size_t)s]);
        std::vector<double> aa((size_t)ns * j.nrecurs), bb((size_t)ns * j.nrecurs);
        ck(gbn_lanczos_sets(ctx, GBN_FP64, ns, set_of_atom.data(), u.data(), assumed.data(), nullptr, j.nrecurs,
                            aa.data(), bb.data()),
           ctx, "gbn_lanczos_sets");
        for (int s = 0; s < ns; ++s) {
            char folder[64];
            if (p.mode == GBN_PDOS_LAYER) snprintf(folder, sizeof folder, "PDOS_layer%02d", sl[(size_t)s]);
            else snprintf(folder, sizeof folder, "PDOS_layer%02d_sub%02d", sl[(size_t)s], ss[(size_t)s]);
            prefix = make_folder(folder, j.prefix);
            kubo_dos_files(ctx, j, prefix, aa.data() + (size_t)s * j.nrecurs, bb.data() + (size_t)s * j.nrecurs);
        }
        // the last set's start vector (KuboInitWFLayerDOS)
        const int last = ns - 1;
        const double nrm = (double)count[(size_t)last] / assumed[(size_t)last];
        const double den = sqrt(assumed[(size_t)last]), fix = (nrm > 0.0 && fabs(nrm - 1.0) > 1.0e-6) ? sqrt(nrm) : 1.0;
        psi.assign((size_t)2 * n, 0.0);
        int64_t k = 0;
        for (int64_t i = 0; i < n; ++i)
            if (set_of_atom[(size_t)i] == last) {
                psi[(size_t)2 * i] = cos(2.0 * kPi * u[(size_t)k]) / den / fix;
                psi[(size_t)2 * i + 1] = sin(2.0 * kPi * u[(size_t)k]) / den / fix;
                ++k;
            }
        a.assign(aa.end() - j.nrecurs, aa.end());
        b.assign(bb.end() - j.nrecurs, bb.end());
        any = true;
        return;
    }
    int64_t cnt = 0;
    ck(gbn_pdos_atoms(&p, n, rat_now.data(), species.data(), layer.data(), ucell.data(), 0, &cnt, nullptr, nullptr),
       nullptr, "gbn_pdos_atoms (atom index out of range?)");
    if (cnt == 0) return;
    std::vector<int64_t> atoms((size_t)cnt);
    std::vector<double> coords((size_t)3 * cnt);
    ck(gbn_pdos_atoms(&p, n, rat_now.data(), species.data(), layer.data(), ucell.data(), cnt, &cnt, atoms.data(),
                      coords.data()),
       nullptr, "gbn_pdos_atoms");
    std::vector<double> aa((size_t)cnt * j.nrecurs), bb((size_t)cnt * j.nrecurs);
    ck(gbn_lanczos_sites(ctx, GBN_FP64, (int32_t)cnt, atoms.data(), nullptr, j.nrecurs, aa.data(), bb.data()), ctx,
       "gbn_lanczos_sites");
    for (int64_t k = 0; k < cnt; ++k) {
        const int64_t i = atoms[(size_t)k];
        if (p.mode != GBN_PDOS_BY_NUMBER) {   // PDOSByNumber writes to the run's own prefix
            char folder[64];
            snprintf(folder, sizeof folder, "PDOS_atom%08lld", (long long)i);
            prefix = make_folder(folder, j.prefix);
            const std::string cpath = "./" + std::string(folder) + "/coords";
            FILE* f = fopen(cpath.c_str(), "w");
            if (!f) die("cannot write " + cpath);
            const double* r = coords.data() + 3 * k;
            if (p.mode == GBN_PDOS_MOIRE_SC1)
                fprintf(f, "%12lld%s%s%12d%12d\n", (long long)i, fortran_ld(r[0]).c_str(), fortran_ld(r[1]).c_str(),
                        species[(size_t)(i - 1)], layer[(size_t)(i - 1)]);
            else
                fprintf(f, "%12lld%s%s%s\n", (long long)i, fortran_ld(r[0]).c_str(), fortran_ld(r[1]).c_str(),
                        fortran_ld(r[2]).c_str());
            fclose(f);
        } else {
            prefix = j.prefix;
        }
        kubo_dos_files(ctx, j, prefix, aa.data() + (size_t)k * j.nrecurs, bb.data() + (size_t)k * j.nrecurs);
    }
    psi.assign((size_t)2 * n, 0.0);
    psi[(size_t)2 * (atoms.back() - 1)] = 1.0;   // KuboInitWFPDOS of the last atom
    a.assign(aa.end() - j.nrecurs, aa.end());
    b.assign(bb.end() - j.nrecurs, bb.end());
    any = true;
}

int run(const Job& j0)
{
    Job j = j0;
    int64_t n = 0;
    ck(gbn_cell_atoms(&j.cell, &n), nullptr, "gbn_cell_atoms");
    std::vector<double> ucell(9), rat((size_t)3 * n);
    std::vector<int32_t> species((size_t)n), layer((size_t)n);
    double twist = 0.0;
    ck(gbn_build_cell(&j.cell, ucell.data(), rat.data(), species.data(), layer.data(), &twist), nullptr,
       "gbn_build_cell");
    const double area = cell_area(ucell.data());
    resolve_fields(j, area);
    printf("grabnes: %lld atoms, cell area %.6f Ang^2, g0 = %.6f eV\n", (long long)n, area, j.g0);
    const Shard shard = shard_from_env();
    if (shard.nranks > 1) {
        const auto units = sweep_units(j);
        long mine = 0;
        for (size_t k = 0; k < units.size(); ++k) mine += shard.mine((long)k) ? 1 : 0;
        printf("grabnes: rank %d of %d, %ld of the %zu units of this job\n", shard.rank, shard.nranks, mine,
               units.size());
        if (mine == 0) return 0;
    }
    gbn_ctx* ctx = nullptr;
    const char* dev = getenv("GRABNES_DEVICE");
    ck(gbn_create(&ctx, dev ? atoi(dev) : 0), nullptr, "gbn_create (no CUDA device?)");
    ck(gbn_set_geometry(ctx, n, rat.data(), species.data(), layer.data(), ucell.data()), ctx, "gbn_set_geometry");
    int32_t maxn = 0;
    int64_t total = 0;
    Tables tab;
    if (j.read_data) {
        tab = read_tables(j, n, ucell, rat);
        maxn = tab.maxn;
        for (int32_t k : tab.nn) total += k;
    } else {
        ck(gbn_neighbours(ctx, j.cut2intra, j.cut2inter, j.second_layer ? 1 : 0, &maxn, &total), ctx, "gbn_neighbours");
        if (j.write_data) write_neigh_files(ctx, n, maxn, rat, species);
    }
    printf("grabnes: %lld neighbour entries (at most %d per atom)\n", (long long)total, maxn);
    std::vector<double> rat_on, rat_hop;
    if (j.moire) {   // the positions the reference's moire routines see after their own conversions
        rat_on = rat;
        ck(gbn_cart_roundtrip(n, ucell.data(), rat_on.data()), nullptr, "gbn_cart_roundtrip");
        rat_hop = rat_on;
        ck(gbn_cart_roundtrip(n, ucell.data(), rat_hop.data()), nullptr, "gbn_cart_roundtrip");
    }
    const std::vector<double>& rat_now = j.moire ? rat_hop : rat;   // the module positions CalcKubo sees
    // Anderson disorder and the start vector draw the same stream (random_seed(PUT=SeedValue) in both)
    std::vector<double> u((size_t)n);
    ck(gbn_rng_uniform(j.seed, n, u.data()), nullptr, "gbn_rng_uniform");
    const bool magfield = !(j.mbi == 0 && j.mbf == 0);
    const std::vector<ShiftUnit> shifts = shift_units(j);
    const bool shift_sweep = shifts.size() > 1;
    // the reference names the folder of every field (or Haldane phase) after the field alone, so that a
    // layer-shift range combined with a field or phase sweep writes all shifts into the same folders
    if (shift_sweep && ((magfield && j.mbi != j.mbf) || j.mphii != j.mphif))
        die("a moireBLShift range combined with a field or Haldane phase sweep writes every shift into the same "
            "folders; run the shifts and the fields as separate jobs");
    for (int k = 0; k < 4; ++k) j.model.tau[k] = shifts[0].tau[k];
    std::vector<double> a((size_t)j.nrecurs), b((size_t)j.nrecurs), psi;
    if (!shift_sweep && magfield && j.mbi != j.mbf && j.pdos.mode == 0 && j.only_dos && !j.read_data && !j.write_data && !j.haldane &&
        j.mphii == j.mphif) {
        // a DOS-only sweep: all fields in one batch from the field-free Hamiltonian, each field's Peierls
        // phases applied on the fly (the reference reseeds, so every field starts from the same vector)
        std::vector<int32_t> fm;
        long unit = 0;
        for (long mb = j.mbi; mb <= j.mbf; mb += j.mstep)
            if (shard.mine(unit++)) fm.push_back((int32_t)mb);
        const int nf = (int)fm.size();
        if (nf == 0) {
            printf("grabnes: rank %d of %d has no field of this sweep\n", shard.rank, shard.nranks);
            gbn_destroy(ctx);
            return 0;
        }
        std::vector<double> uu((size_t)nf * n), aa((size_t)nf * j.nrecurs), bb((size_t)nf * j.nrecurs);
        for (int f = 0; f < nf; ++f) std::copy(u.begin(), u.end(), uu.begin() + (size_t)f * n);
        ck(gbn_assemble(ctx, &j.model, j.moire ? rat_on.data() : nullptr, j.moire ? rat_hop.data() : nullptr,
                        j.model.anderson ? u.data() : nullptr),
           ctx, "gbn_assemble");
        ck(gbn_lanczos_fields(ctx, GBN_FP64, nf, fm.data(), 1, uu.data(), nullptr, j.nrecurs, aa.data(), bb.data()),
           ctx, "gbn_lanczos_fields");
        printf("grabnes: %d fields in one batch\n", nf);
        for (int f = 0; f < nf; ++f) {
            const double bmag = fm[(size_t)f] * kFluxQuantum / (area * 1.0e-20);
            char folder[64];
            snprintf(folder, sizeof folder, "m%05d_B%.4f", fm[(size_t)f], bmag);
            if (mkdir(folder, 0755) != 0 && errno != EEXIST) die(std::string("cannot create folder ") + folder);
            const std::string prefix = std::string("./") + folder + "/" + j.prefix;
            printf("grabnes: field %d of %ld..%ld, %.5f T, files in %s\n", fm[(size_t)f], j.mbi, j.mbf, bmag, folder);
            kubo_dos_files(ctx, j, prefix, aa.data() + (size_t)f * j.nrecurs, bb.data() + (size_t)f * j.nrecurs);
            if (j.polynomials) {   // <prefix>.cn.dat only: Calculate.OnlyDOS stops before the evolution
                a.assign(aa.begin() + (size_t)f * j.nrecurs, aa.begin() + (size_t)(f + 1) * j.nrecurs);
                b.assign(bb.begin() + (size_t)f * j.nrecurs, bb.begin() + (size_t)(f + 1) * j.nrecurs);
                time_evolution(ctx, j, psi, a, b, prefix, n);
            }
        }
        gbn_destroy(ctx);
        return 0;
    }
    const bool hsweep = j.mphii != j.mphif;   // HaldPhaseInit: a Haldane phase sweep
    long unit = -1;
    for (size_t sh = 0; sh < shifts.size(); ++sh) {   // moireBLShift.Calc: HamOnSite and HamHopping per shift
    std::string base = j.prefix;
    if (shift_sweep) {
        if (!shard.mine((long)sh)) continue;   // another rank's shift
        for (int k = 0; k < 4; ++k) j.model.tau[k] = shifts[sh].tau[k];
        printf("grabnes: layer shift %zu of 0..%zu (tauX1 %.4f tauY1 %.4f tauX2 %.4f tauY2 %.4f)\n", sh,
               shifts.size() - 1, shifts[sh].tau[0], shifts[sh].tau[1], shifts[sh].tau[2], shifts[sh].tau[3]);
        base = make_folder(shifts[sh].folder, j.prefix);
    }
    for (long mb = j.mbi; mb <= j.mbf; mb += (magfield ? j.mstep : 1))
    for (long mphi = j.mphii; mphi <= j.mphif; mphi += j.mphistep) {
        if (!shift_sweep && !shard.mine(++unit)) {   // another rank's unit
            if (!magfield && !hsweep) break;
            continue;
        }
        std::string prefix = base;
        if (magfield && j.mbi != j.mbf) {
            const double bmag = mb * kFluxQuantum / (area * 1.0e-20);
            char folder[64];
            snprintf(folder, sizeof folder, "m%05ld_B%.4f", mb, bmag);
            if (mkdir(folder, 0755) != 0 && errno != EEXIST) die(std::string("cannot create folder ") + folder);
            prefix = std::string("./") + folder + "/" + j.prefix;
            printf("grabnes: field %ld of %ld..%ld, %.5f T, files in %s\n", mb, j.mbi, j.mbf, bmag, folder);
        }
        // HaldPhaseValue (magf.F90:213-250): the phase of step mphi, and its folder (named like a field's)
        double hphase = 0.0;
        if (j.hal_mode == 1) hphase = j.hal_setfluxq ? 2.0 * kPi * j.hal_flux / 1.0471975512 : 2.0 * kPi * j.hal_flux / kFluxQuantum;
        else if (j.hal_mode == 2) hphase = j.hal_phase;
        else if (j.hal_mode == 3 && hsweep) hphase = 1.0 / (double)(j.mphif - j.mphii) * (double)mphi * 2.0 * kPi;
        if (hsweep) {
            char folder[64];
            snprintf(folder, sizeof folder, "m%05ld_B%.4f", mphi, hphase);
            if (mkdir(folder, 0755) != 0 && errno != EEXIST) die(std::string("cannot create folder ") + folder);
            prefix = std::string("./") + folder + "/" + j.prefix;
            printf("grabnes: Haldane phase step %ld of %ld..%ld, %.6f rad, files in %s\n", mphi, j.mphii, j.mphif, hphase,
                   folder);
        }
        if (j.hal_opposite) hphase = -hphase;
        if (j.read_data) {   // the hoppings of generate.s for every field, then its phases
            ck(gbn_load_hamiltonian(ctx, n, tab.maxn, tab.nn.data(), tab.nl.data(), tab.hop.data(), tab.h0.data()), ctx,
               "gbn_load_hamiltonian");
            ck(gbn_set_images(ctx, tab.nc.data()), ctx, "gbn_set_images");
            ck(gbn_set_neighd(ctx, tab.nd.data()), ctx, "gbn_set_neighd");
        } else {
            ck(gbn_assemble(ctx, &j.model, j.moire ? rat_on.data() : nullptr, j.moire ? rat_hop.data() : nullptr,
                            j.model.anderson ? u.data() : nullptr),
               ctx, "gbn_assemble");
        }
        if (magfield) {
            const double bmag = mb * kFluxQuantum / (area * 1.0e-20);
            ck(gbn_peierls(ctx, bmag * kPi / kFluxQuantum), ctx, "gbn_peierls");
        }
        if (j.haldane) ck(gbn_haldane(ctx, j.cell.aG, j.hal_t2, hphase, j.hal_paper ? 1 : 0, j.hal_mask), ctx, "gbn_haldane");
        if (!j.read_data) check_hamiltonian(ctx, j);
        if (j.write_data && !j.read_data) write_ham_files(ctx, prefix, n, maxn, rat_now, species, layer, ucell.data(),
                                                        j.model.second_moire != 0);
        bool any = true;
        if (j.pdos.mode == 0) {   // KuboInitWF + KuboDOS
            ck(gbn_lanczos_phases(ctx, GBN_FP64, 1, u.data(), nullptr, j.nrecurs, a.data(), b.data()), ctx,
               "gbn_lanczos_phases");
            kubo_dos_files(ctx, j, prefix, a.data(), b.data());
            psi.assign((size_t)2 * n, 0.0);
            const double isn = 1.0 / sqrt((double)n);
            for (int64_t i = 0; i < n; ++i) {
                psi[(size_t)2 * i] = cos(2.0 * kPi * u[(size_t)i]) * isn;
                psi[(size_t)2 * i + 1] = sin(2.0 * kPi * u[(size_t)i]) * isn;
            }
        } else {
            pdos_pass(ctx, j, n, rat_now, species, layer, ucell, psi, a, b, prefix, any);
        }
        if (j.polynomials || !j.only_dos) {
            if (any) time_evolution(ctx, j, psi, a, b, prefix, n);
            else printf("grabnes: the PDOS selection is empty: no time evolution\n");
        }
        if (!magfield && !hsweep) break;
    }
    }
    gbn_destroy(ctx);
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    bool print = false;
    std::string path = "Gendata.in";
    for (int k = 1; k < argc; ++k) {
        if (strcmp(argv[k], "--print-job") == 0) print = true;
        else path = argv[k];
    }
    Input in;
    in.load(path);
    const Job j = job_from_input(in);
    if (print) {
        print_job(j);
        return 0;
    }
    return run(j);
}
