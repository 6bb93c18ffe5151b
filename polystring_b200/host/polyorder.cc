// polyorder.cc -- implementation of the host classes in polyorder.h.
#include "polyorder.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <random>
#include <sstream>

namespace polyorder {

namespace {

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return s;
}
std::string upper(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::toupper(c); });
    return s;
}
std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}
void check(int rc) {
    if (rc != PS_OK) throw std::runtime_error(std::string("polystring_b200: ") + ps_last_error());
}

}  // namespace

// ---------------------------------------------------------------------------
// Config (INI sections/keys are case-insensitive, as SimpleIni's default)
// ---------------------------------------------------------------------------
Config::Config(const std::string& file) {
    std::ifstream in(file);
    if (!in) throw std::runtime_error("cannot open config file " + file);
    size_t slash = file.find_last_of('/');
    dir_ = slash == std::string::npos ? std::string("./") : file.substr(0, slash + 1);
    std::string line, section;
    while (std::getline(in, line)) {
        std::string t = trim(line);
        if (t.empty() || t[0] == '#' || t[0] == ';') continue;
        if (t[0] == '[') {
            size_t e = t.find(']');
            section = lower(trim(t.substr(1, e == std::string::npos ? std::string::npos : e - 1)));
            continue;
        }
        size_t eq = t.find('=');
        if (eq == std::string::npos) continue;
        kv_[section][lower(trim(t.substr(0, eq)))] = trim(t.substr(eq + 1));
    }
}

std::string Config::get_string(const std::string& section, const std::string& key, const std::string& def) const {
    auto s = kv_.find(lower(section));
    if (s == kv_.end()) return def;
    auto k = s->second.find(lower(key));
    if (k == s->second.end() || k->second.empty()) return def;
    return k->second;
}

double Config::get_double(const std::string& section, const std::string& key, double def) const {
    std::string v = get_string(section, key);
    return v.empty() ? def : std::stod(v);
}

int Config::get_integer(const std::string& section, const std::string& key, int def) const {
    std::string v = get_string(section, key);
    return v.empty() ? def : (int)std::stol(v);
}

bool Config::get_bool(const std::string& section, const std::string& key, bool def) const {
    std::string v = lower(get_string(section, key));
    if (v.empty()) return def;
    return v == "true" || v == "1" || v == "yes" || v == "on";
}

// Python-style lists "[a, b, c]" (Config.cc:1549-1624)
std::vector<double> Config::get_list(const std::string& section, const std::string& key) const {
    std::string v = get_string(section, key);
    std::vector<double> out;
    std::string cur;
    for (char ch : v) {
        if (ch == '[' || ch == ']' || ch == ',' || ch == ' ') {
            if (!trim(cur).empty()) out.push_back(std::stod(trim(cur)));
            cur.clear();
        } else {
            cur += ch;
        }
    }
    if (!trim(cur).empty()) out.push_back(std::stod(trim(cur)));
    return out;
}

void Config::set(const std::string& section, const std::string& key, double v) {
    std::ostringstream os;
    os << std::setprecision(17) << v;
    kv_[lower(section)][lower(key)] = os.str();
}

// Config::algo_mde_type (Config.cc:1099-1111)
AlgorithmMDEType Config::algo_mde_type() const {
    std::string t = upper(get_string("Algorithm_MDE", "algorithm"));
    if (t == "PSEUDOSPECTRAL" || t == "OS2" || t == "OS") return AlgorithmMDEType::OS2;
    if (t == "RQM4" || t == "OS4") return AlgorithmMDEType::RQM4;
    return AlgorithmMDEType::ETDRK4;
}

// Config::algo_scft_type (Config.cc:1219-1235)
AlgorithmSCFTType Config::algo_scft_type() const {
    std::string t = upper(get_string("Algorithm_SCFT", "algorithm"));
    if (t == "ANDERSON" || t == "ANDERSON_MIXING" || t == "ANDERSON MIXING") return AlgorithmSCFTType::ANDERSON;
    return AlgorithmSCFTType::EM;
}

// Config::algo_contour_integration_type (Config.cc:1495-1505)
AlgorithmContourType Config::algo_contour_integration_type() const {
    std::string t = upper(get_string("Algorithm_Contour_Integration", "algorithm"));
    if (t == "TRAPEZOIDAL" || t == "TRAP" || t == "TRAPE" || t == "TRAPZ") return AlgorithmContourType::TRAPEZOIDAL;
    return AlgorithmContourType::SIMPSON;
}

// Config::algo_cell_optimization_type (Config.cc:1335-1349)
AlgorithmCellType Config::algo_cell_optimization_type() const {
    std::string t = upper(get_string("Algorithm_Cell_Optimization", "algorithm"));
    if (t == "MANUAL" || t == "BATCH") return AlgorithmCellType::MANUAL;
    if (t == "BRENT" || t == "BRENT METHOD" || t == "NEWTON") return AlgorithmCellType::BRENT;
    return AlgorithmCellType::SINGLE;
}

// Config::get_grid_init_type (Config.cc:977-992)
GridInitType Config::get_grid_init_type() const {
    std::string t = upper(get_string("Grid", "gridInitType"));
    if (t == "CONST" || t == "CONSTANT") return GridInitType::CONSTANT_INIT;
    if (t == "DATA") return GridInitType::DATA_INIT;
    if (t == "FILE") return GridInitType::FILE_INIT;
    if (t == "PATTERN") return GridInitType::PATTERN_INIT;
    return GridInitType::RANDOM_INIT;
}

// ---------------------------------------------------------------------------
// UnitCell (crystal system names of Config::get_crystal_system_type, :518-547)
// ---------------------------------------------------------------------------
UnitCell::UnitCell(const Config& cfg) {
    std::memset(&cell_, 0, sizeof(cell_));
    cell_.dim = cfg.dim();
    std::string t = upper(cfg.crystal_system());
    int sys = -1;
    if (t == "LAM" || t == "LAMELLAR" || t == "LAMELLA" || t == "LAMELLAE") sys = PS_CELL_LAMELLAR;
    else if (t == "SQUARE" || t == "SQ") sys = PS_CELL_SQUARE;
    else if (t == "RECT" || t == "RECTANGLE" || t == "RECTANGULAR") sys = PS_CELL_RECTANGULAR;
    else if (t == "HEX" || t == "HEXAGONAL" || t == "HEXGON") sys = cell_.dim == 3 ? PS_CELL_HEXAGONAL3 : PS_CELL_HEXAGONAL2;
    else if (t == "OBLIQUE" || t == "OB") sys = PS_CELL_OBLIQUE;
    else if (t == "CUBIC" || t == "CUBE") sys = PS_CELL_CUBIC;
    else if (t == "TETRAGONAL" || t == "TETRAGON") sys = PS_CELL_TETRAGONAL;
    else if (t == "ORTHORHOMBIC") sys = PS_CELL_ORTHORHOMBIC;
    else if (t == "TRIGONAL") sys = PS_CELL_TRIGONAL;
    else if (t == "MONOCLINIC") sys = PS_CELL_MONOCLINIC;
    else if (t == "TRICLINIC") sys = PS_CELL_TRICLINIC;
    if (sys < 0) throw std::runtime_error("unknown crystal system type: " + cfg.crystal_system());
    cell_.system = sys;
    cell_.a = cfg.a();
    cell_.b = cfg.b();
    cell_.c = cfg.c();
    cell_.alpha = cfg.get_double("UnitCell", "alpha");
    cell_.beta = cfg.get_double("UnitCell", "beta");
    cell_.gamma = cfg.get_double("UnitCell", "gamma");
    if (sys == PS_CELL_SQUARE || sys == PS_CELL_HEXAGONAL2) cell_.b = cell_.a;
    if (sys == PS_CELL_CUBIC) { cell_.b = cell_.a; cell_.c = cell_.a; }
    if (sys == PS_CELL_TETRAGONAL || sys == PS_CELL_HEXAGONAL3) cell_.b = cell_.a;
}

// ---------------------------------------------------------------------------
// Grid and MAT-file v5
// ---------------------------------------------------------------------------
double Grid::quadrature() const {
    double s = 0.0;
    for (double v : data_) s += v;
    return s / (double)data_.size();
}

namespace {
constexpr uint32_t miINT8 = 1, miINT32 = 5, miUINT32 = 6, miDOUBLE = 9, miMATRIX = 14;

struct Rd {
    const std::vector<char>& b;
    size_t off;
    uint32_t u32(size_t o) const { uint32_t v; std::memcpy(&v, b.data() + o, 4); return v; }
};

// one data element: type, byte count, payload offset, total size (padded)
void tag(const std::vector<char>& b, size_t off, uint32_t& type, uint32_t& nbytes, size_t& data, size_t& total) {
    uint32_t w0;
    std::memcpy(&w0, b.data() + off, 4);
    if (w0 >> 16) {   // small data element
        type = w0 & 0xffff;
        nbytes = w0 >> 16;
        data = off + 4;
        total = 8;
    } else {
        type = w0;
        std::memcpy(&nbytes, b.data() + off + 4, 4);
        data = off + 8;
        total = 8 + ((nbytes + 7) / 8) * 8;
    }
}

// The values of a numeric data element as doubles.  MATLAB stores an array
// in the smallest type that holds its values exactly (a double array of
// small integers as miUINT8, for instance), whatever the array's class, and
// reads it back as the class; so every numeric storage type is converted.
bool mat_numeric(uint32_t type, const char* p, uint32_t nbytes, std::vector<double>& v) {
    auto conv = [&](auto zero) {
        using T = decltype(zero);
        const size_t n = nbytes / sizeof(T);
        v.resize(n);
        for (size_t i = 0; i < n; i++) {
            T x;
            std::memcpy(&x, p + i * sizeof(T), sizeof(T));
            v[i] = (double)x;
        }
        return true;
    };
    switch (type) {
    case 1: return conv(int8_t());
    case 2: return conv(uint8_t());
    case 3: return conv(int16_t());
    case 4: return conv(uint16_t());
    case 5: return conv(int32_t());
    case 6: return conv(uint32_t());
    case 7: return conv(float());
    case 9: return conv(double());
    case 12: return conv(int64_t());
    case 13: return conv(uint64_t());
    }
    return false;
}
}  // namespace

std::vector<double> mat_read(const std::string& file, const std::string& name, std::vector<int>* dims_out) {
    std::ifstream in(file, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open MAT-file " + file);
    std::vector<char> b((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    if (b.size() < 128) throw std::runtime_error("truncated MAT-file " + file);
    size_t off = 128;
    while (off + 8 <= b.size()) {
        uint32_t type, nb;
        size_t data, total;
        tag(b, off, type, nb, data, total);
        if (data + nb > b.size()) throw std::runtime_error("truncated MAT-file " + file);
        if (type == 15) throw std::runtime_error("compressed MAT-files are not supported: " + file);
        if (type == miMATRIX) {
            size_t p = data, end = data + nb;
            uint32_t t, n;
            size_t d, tot;
            tag(b, p, t, n, d, tot);          // array flags
            p += tot;
            tag(b, p, t, n, d, tot);          // dimensions
            std::vector<int> dims(n / 4);
            for (size_t i = 0; i < dims.size(); i++) { int32_t v; std::memcpy(&v, b.data() + d + 4 * i, 4); dims[i] = v; }
            p += tot;
            tag(b, p, t, n, d, tot);          // name
            std::string vname(b.data() + d, n);
            p += tot;
            if (vname == name) {
                tag(b, p, t, n, d, tot);      // real part
                if (p + tot > end) throw std::runtime_error("truncated variable " + name + " in " + file);
                std::vector<double> v;
                if (!mat_numeric(t, b.data() + d, n, v))
                    throw std::runtime_error("variable " + name + " of " + file + " has no numeric real part");
                if (dims_out) *dims_out = dims;
                return v;
            }
        }
        off += total;
    }
    throw std::runtime_error("variable " + name + " not found in " + file);
}

void mat_write(const std::string& file, const std::map<std::string, std::pair<std::vector<int>, std::vector<double>>>& vars) {
    std::ofstream out(file, std::ios::binary);
    if (!out) throw std::runtime_error("cannot write MAT-file " + file);
    char hdr[128];
    std::memset(hdr, ' ', 116);
    std::snprintf(hdr, 116, "MATLAB 5.0 MAT-file, written by polystring_b200");
    hdr[std::strlen(hdr)] = ' ';
    std::memset(hdr + 116, 0, 8);
    uint16_t ver = 0x0100;
    std::memcpy(hdr + 124, &ver, 2);
    hdr[126] = 'I';
    hdr[127] = 'M';
    out.write(hdr, 128);
    auto w32 = [&](uint32_t v) { out.write(reinterpret_cast<const char*>(&v), 4); };
    for (const auto& kv : vars) {
        const std::string& nm = kv.first;
        const std::vector<int>& dims = kv.second.first;
        const std::vector<double>& v = kv.second.second;
        uint32_t name_pad = ((uint32_t)nm.size() + 7) / 8 * 8;
        uint32_t dim_bytes = 4 * (uint32_t)dims.size(), dim_pad = (dim_bytes + 7) / 8 * 8;
        uint32_t body = 16 + 8 + dim_pad + 8 + name_pad + 8 + 8 * (uint32_t)v.size();
        w32(miMATRIX); w32(body);
        w32(miUINT32); w32(8); w32(6); w32(0);                  // mxDOUBLE_CLASS
        w32(miINT32); w32(dim_bytes);
        for (int d : dims) w32((uint32_t)d);
        for (uint32_t i = dim_bytes; i < dim_pad; i++) out.put(0);
        w32(miINT8); w32((uint32_t)nm.size());
        out.write(nm.data(), nm.size());
        for (uint32_t i = (uint32_t)nm.size(); i < name_pad; i++) out.put(0);
        w32(miDOUBLE); w32(8 * (uint32_t)v.size());
        out.write(reinterpret_cast<const char*>(v.data()), 8 * v.size());
    }
}

// MAT stores column-major (Fortran) order; the grid is row-major (z fastest)
void Grid::load_mat(const std::string& file, const std::string& name) {
    std::vector<int> dims;
    std::vector<double> v = mat_read(file, name, &dims);
    if ((long)v.size() != size()) throw std::runtime_error("size of " + name + " in " + file + " does not match the grid");
    for (int i = 0; i < Lx_; i++)
        for (int j = 0; j < Ly_; j++)
            for (int k = 0; k < Lz_; k++)
                data_[((size_t)i * Ly_ + j) * Lz_ + k] = v[((size_t)k * Ly_ + j) * Lx_ + i];
}

// ---------------------------------------------------------------------------
// updaters
// ---------------------------------------------------------------------------
PropagatorUpdater::PropagatorUpdater(int scheme, const UnitCell& uc, int Lx, int Ly, int Lz, double ds) {
    check(ps_updater_create(scheme, &uc.c_cell(), Lx, Ly, Lz, ds, &h_));
}

PropagatorUpdater::PropagatorUpdater(const PropagatorUpdater& rhs) : Updater(rhs) {
    check(ps_updater_clone(rhs.h_, &h_));
}

PropagatorUpdater::~PropagatorUpdater() { ps_updater_destroy(h_); }

void PropagatorUpdater::solve(Propagator& q, const Grid& w) { check(ps_updater_solve(h_, w.data(), q.qs(), q.len())); }

void Propagator::set_head(const double* u) { std::memcpy(qs_.data(), u, sizeof(double) * size()); }

double Propagator::Q(int s) const {
    const double* p = qs_.data() + (size_t)s * size();
    double acc = 0.0;
    for (long i = 0; i < size(); i++) acc += p[i];
    return acc / (double)size();
}

void DensityUpdater::solve(std::vector<double>& data, const Propagator& q, const Propagator& qc, double cc) const {
    check(ps_density_solve(rule_, q.qs(), qc.qs(), q.len(), q.size(), q.ds(), cc, data.data()));
}

void Density::update(const Propagator& q, const Propagator& qc, double cc) {
    if (up_) {
        up_->solve(vec(), q, qc, cc);
    } else {
        check(ps_density_solve(PS_CONTOUR_TRAPEZOID, q.qs(), qc.qs(), q.len(), q.size(), q.ds(), cc, data()));
    }
}

// ---------------------------------------------------------------------------
// Model_AB
// ---------------------------------------------------------------------------
Model_AB::Model_AB(const Config& cfg) : Lx_(cfg.Lx()), Ly_(cfg.Ly()), Lz_(cfg.Lz()) {
    std::string confine = upper(cfg.get_string("Grid", "confine_geometry", "NONE"));
    if (!(confine == "NONE" || confine.empty()))
        throw std::runtime_error("only periodic cells (confine_geometry = None) are provided by the B200 backend");
    ps_model_ab_params& p = p_;
    std::memset(&p, 0, sizeof(p));
    p.dim = cfg.dim();
    p.Lx = Lx_; p.Ly = Ly_; p.Lz = Lz_;
    p.cell = UnitCell(cfg).c_cell();
    std::vector<double> Ms = cfg.Ms();
    if (Ms.size() < 2) throw std::runtime_error("[Algorithm_MDE] Ms needs two entries");
    p.sA = (int)Ms[0];
    p.sB = (int)Ms[1];
    p.chiN = cfg.chiN();
    std::vector<double> lam = cfg.lam();
    if (lam.size() < 3) throw std::runtime_error("[Algorithm_SCFT] lam needs three entries");
    p.lamA = lam[0]; p.lamB = lam[1]; p.lamYita = lam[2];
    // Model_AB::init_propagator (Model_AB.cc:740-790): ETDRK4 is Etdrk4_PBC (Cox-Matthews)
    switch (cfg.algo_mde_type()) {
    case AlgorithmMDEType::OS2: p.mde = PS_MDE_OS2; break;
    case AlgorithmMDEType::ETDRK4: p.mde = PS_MDE_ETDRK4; break;
    default: p.mde = PS_MDE_RQM4; break;
    }
    p.etdrk4_M = cfg.etdrk4_M();
    p.scft = cfg.algo_scft_type() == AlgorithmSCFTType::ANDERSON ? PS_SCFT_ANDERSON : PS_SCFT_EM;
    p.n_anderson = cfg.n_Anderson_mixing();
    p.compressible = cfg.is_compressible() ? 1 : 0;
    p.contour = cfg.algo_contour_integration_type() == AlgorithmContourType::SIMPSON ? 1 : 0;
    check(ps_model_ab_create(&p, &h_));
    // Model_AB::init_field (Model_AB.cc:687-711)
    const long M = (long)Lx_ * Ly_ * Lz_;
    std::vector<double> wA(M), wB(M);
    switch (cfg.get_grid_init_type()) {
    case GridInitType::FILE_INIT: {
        Grid a(Lx_, Ly_, Lz_), b(Lx_, Ly_, Lz_);
        std::string f = cfg.field_data_file();
        if (!f.empty() && f[0] != '/') f = cfg.dir() + f;
        a.load_mat(f, "wA");
        b.load_mat(f, "wB");
        wA = a.vec();
        wB = b.vec();
        break;
    }
    case GridInitType::CONSTANT_INIT:
        std::fill(wA.begin(), wA.end(), 0.5);
        std::fill(wB.begin(), wB.end(), 0.5);
        break;
    default: {
        // uniform [0, 1) from the seed (the reference's generator is not
        // reproducible here; Grid.cc:713-725 uses the same range)
        std::mt19937_64 gen((uint64_t)cfg.seed());
        std::uniform_real_distribution<double> u(0.0, 1.0);
        for (long i = 0; i < M; i++) wA[i] = u(gen);
        for (long i = 0; i < M; i++) wB[i] = u(gen);
        break;
    }
    }
    set_fields(wA, wB);
}

Model_AB::~Model_AB() { ps_model_ab_destroy(h_); }

void Model_AB::set_fields(const std::vector<double>& wA, const std::vector<double>& wB) {
    check(ps_model_ab_set_fields(h_, wA.data(), wB.data()));
}

void Model_AB::reset_cell(const Config& cfg) {
    std::vector<double> wA = field(PS_FIELD_WA), wB = field(PS_FIELD_WB);
    ps_model_ab* h = nullptr;
    ps_model_ab_params p = p_;
    p.cell = UnitCell(cfg).c_cell();
    check(ps_model_ab_create(&p, &h));
    ps_model_ab_destroy(h_);
    h_ = h;
    p_ = p;
    set_fields(wA, wB);
}

std::vector<double> Model_AB::lengths() const {
    const int d = p_.dim;
    return {p_.cell.a, d >= 2 ? p_.cell.b : 0.0, d >= 3 ? p_.cell.c : 0.0};
}

bool Model_AB::has_stress() const { return p_.mde == PS_MDE_RQM4 && p_.dim >= 2; }

std::vector<double> Model_AB::stress() const {
    std::vector<double> s(3, 0.0);
    check(ps_model_ab_stress(h_, s.data()));
    return s;
}

void Model_AB::update() { check(ps_model_ab_update(h_, 1)); }
void Model_AB::update(int n) { check(ps_model_ab_update(h_, n)); }

double Model_AB::H() const {
    double H, Hw, Hs;
    check(ps_model_ab_H(h_, &H, &Hw, &Hs));
    return H;
}
double Model_AB::Hw() const {
    double H, Hw, Hs;
    check(ps_model_ab_H(h_, &H, &Hw, &Hs));
    return Hw;
}
double Model_AB::Hs() const {
    double H, Hw, Hs;
    check(ps_model_ab_H(h_, &H, &Hw, &Hs));
    return Hs;
}
double Model_AB::residual_error() const {
    double r;
    check(ps_model_ab_residual(h_, &r));
    return r;
}
double Model_AB::Q() const {
    double q;
    check(ps_model_ab_Q(h_, &q));
    return q;
}

std::vector<double> Model_AB::field(int which) const {
    std::vector<double> out((size_t)Lx_ * Ly_ * Lz_);
    check(ps_model_ab_get(h_, which, out.data()));
    return out;
}

// Model_AB::display (Model_AB.cc:383-427), the lines that concern this path
void Model_AB::display() const {
    double H, Hw, Hs;
    check(ps_model_ab_H(h_, &H, &Hw, &Hs));
    std::cout << std::fixed << std::setprecision(6) << "\tH    = " << H << " = " << Hw << " + " << Hs << "\n";
    std::cout << std::scientific << std::setprecision(2) << "\tQ_qB = " << Q() << "\n"
              << "\tResidual Error    = " << residual_error() << "\n";
    std::cout.unsetf(std::ios::floatfield);
}

// fields and densities as MAT-file v5 variables (Model_AB::save, :440-469)
void Model_AB::save(const std::string& file) {
    std::vector<int> dims = {Lx_, Ly_, Lz_};
    auto colmajor = [&](const std::vector<double>& v) {
        std::vector<double> o(v.size());
        for (int i = 0; i < Lx_; i++)
            for (int j = 0; j < Ly_; j++)
                for (int k = 0; k < Lz_; k++)
                    o[((size_t)k * Ly_ + j) * Lx_ + i] = v[((size_t)i * Ly_ + j) * Lz_ + k];
        return o;
    };
    std::map<std::string, std::pair<std::vector<int>, std::vector<double>>> vars;
    vars["wA"] = {dims, colmajor(field(PS_FIELD_WA))};
    vars["wB"] = {dims, colmajor(field(PS_FIELD_WB))};
    vars["phiA"] = {dims, colmajor(field(PS_FIELD_PHIA))};
    vars["phiB"] = {dims, colmajor(field(PS_FIELD_PHIB))};
    mat_write(file, vars);
}

// ---------------------------------------------------------------------------
// scft
// ---------------------------------------------------------------------------
void scft::run() {
    switch (cfg_.algo_cell_optimization_type()) {
    case AlgorithmCellType::BRENT:
        optimize_cell();
        break;
    case AlgorithmCellType::MANUAL: {
        std::vector<double> lo = cfg_.get_list("Algorithm_Cell_Optimization", "batch_cell_min");
        std::vector<double> st = cfg_.get_list("Algorithm_Cell_Optimization", "batch_cell_step");
        std::vector<double> hi = cfg_.get_list("Algorithm_Cell_Optimization", "batch_cell_max");
        lo.resize(3, 0.0); st.resize(3, 1.0); hi.resize(3, 0.0);
        for (int i = 0; i < 3; i++) if (st[i] <= 0) st[i] = 1.0;
        for (double a = lo[0]; a <= hi[0] + 1e-12; a += st[0])
            for (double b = lo[1]; b <= hi[1] + 1e-12; b += st[1])
                for (double c = lo[2]; c <= hi[2] + 1e-12; c += st[2]) {
                    cfg_.a(a); cfg_.b(b); cfg_.c(c);
                    Model_AB* m = static_cast<Model_AB*>(m_);
                    if (nsolve_ > 0) m->reset_cell(cfg_);
                    relax();
                    std::vector<double> l = m->lengths();
                    trace_.push_back({l[0], l[1], l[2], Hlast_});
                    nsolve_++;
                }
        break;
    }
    default:
        relax();
    }
}

void scft::update_cell(double a, double& b, double& c) const {
    std::vector<double> lo = cfg_.get_list("Algorithm_Cell_Optimization", "batch_cell_min");
    lo.resize(3, 0.0);
    const double a0 = lo[0];
    b = lo[1];
    c = lo[2];
    auto regular = [&](const char* key) {
        std::string t = upper(cfg_.get_string("Grid", key, "REGULAR"));
        return t.empty() || t == "REGULAR";
    };
    if (cfg_.dim() == 2 && regular("grid_type_y")) b = lo[1] * (a / a0);
    if (cfg_.dim() == 3 && regular("grid_type_z")) {
        b = lo[1] * (a / a0);
        c = lo[2] * (a / a0);
    }
}

double scft::solve_cell(double a, double* dFda) {
    double b, c;
    update_cell(a, b, c);
    Model_AB* m = static_cast<Model_AB*>(m_);
    const bool same = nsolve_ == 0 && a == cfg_.a();
    cfg_.a(a); cfg_.b(b); cfg_.c(c);
    if (!same) m->reset_cell(cfg_);
    const int before = iter_;
    relax();
    iter_ += before;
    std::vector<double> l = m->lengths();
    trace_.push_back({l[0], l[1], l[2], Hlast_});
    nsolve_++;
    if (dFda) {
        // every length scales with a (update_cell), so dF/da = sum_i s_i l_i / a
        std::vector<double> s = m->stress();
        *dFda = (s[0] * l[0] + s[1] * l[1] + s[2] * l[2]) / a;
    }
    if (cfg_.is_display())
        std::cout << "cell a = " << a << "  F = " << std::setprecision(12) << Hlast_
                  << (dFda ? "  dF/da = " + std::to_string(*dFda) : std::string()) << std::setprecision(6) << "\n";
    return Hlast_;
}

// BRENT cell optimisation.  The reference brackets the minimum of F(a) from
// batch_cell_min with steps of batch_cell_step and the golden ratio, then
// runs Brent's parabolic / golden-section minimiser to the relative
// tolerance tol_cell (scft.cc:124-309), one converged SCFT solve per trial.
// Here every solve also yields dF/da from the adjoint stress at the converged
// fields, so the minimum is found as the root of dF/da: the sign change is
// bracketed the same way, then Brent-Dekker root finding (inverse quadratic
// interpolation with bisection safeguards; R. P. Brent, Algorithms for
// Minimization without Derivatives, 1973, ch. 4) narrows it to tol_cell |a|.
// Without a stress (1D grids, OS2) the same bracket feeds Brent's
// derivative-free minimiser (ibid., ch. 5) on F alone.
void scft::optimize_cell() {
    std::vector<double> lo = cfg_.get_list("Algorithm_Cell_Optimization", "batch_cell_min");
    std::vector<double> st = cfg_.get_list("Algorithm_Cell_Optimization", "batch_cell_step");
    if (lo.empty() || st.empty()) throw std::runtime_error("BRENT needs batch_cell_min and batch_cell_step");
    const double tol = cfg_.get_double("Algorithm_Cell_Optimization", "tol_cell", 1e-4);
    const int max_solves = std::max(4, cfg_.get_integer("Algorithm_Cell_Optimization", "max_iter_cell", 30) + 10);
    const double GOLD = 1.618034, CGOLD = 0.3819660;
    Model_AB* m = static_cast<Model_AB*>(m_);
    const bool grad = m->has_stress();
    std::map<double, double> Fat;   // F of every solved a
    auto F_of = [&](double a, double* g) {
        double F = solve_cell(a, g);
        Fat[a] = F;
        return F;
    };
    double a0 = lo[0], h = st[0];
    if (grad) {
        double g0, g1;
        F_of(a0, &g0);
        if (g0 > 0) h = -h;              // F rises to the right: search to the left
        double a1 = a0 + h;
        F_of(a1, &g1);
        while ((g0 < 0) == (g1 < 0) && g1 != 0.0) {
            if (nsolve_ >= max_solves) throw std::runtime_error("BRENT: no sign change of dF/da was bracketed");
            a0 = a1; g0 = g1; h *= GOLD;
            a1 = a0 + h;
            if (a1 <= 0) throw std::runtime_error("BRENT: the bracket left the positive cell lengths");
            F_of(a1, &g1);
        }
        // Brent-Dekker on g(a) = dF/da over [a0, a1]
        double xa = a0, fa = g0, xb = a1, fb = g1, xc = xa, fc = fa, d = xb - xa, e = d;
        while (true) {
            if ((fb > 0) == (fc > 0)) { xc = xa; fc = fa; d = e = xb - xa; }
            if (std::fabs(fc) < std::fabs(fb)) { xa = xb; xb = xc; xc = xa; fa = fb; fb = fc; fc = fa; }
            const double tol1 = 2.0 * 2.2e-16 * std::fabs(xb) + 0.5 * tol * std::fabs(xb);
            const double xm = 0.5 * (xc - xb);
            if (std::fabs(xm) <= tol1 || fb == 0.0 || nsolve_ >= max_solves) break;
            if (std::fabs(e) >= tol1 && std::fabs(fa) > std::fabs(fb)) {
                double s = fb / fa, p, q;
                if (xa == xc) {
                    p = 2.0 * xm * s;
                    q = 1.0 - s;
                } else {
                    double qq = fa / fc, r = fb / fc;
                    p = s * (2.0 * xm * qq * (qq - r) - (xb - xa) * (r - 1.0));
                    q = (qq - 1.0) * (r - 1.0) * (s - 1.0);
                }
                if (p > 0) q = -q;
                p = std::fabs(p);
                if (2.0 * p < std::min(3.0 * xm * q - std::fabs(tol1 * q), std::fabs(e * q))) {
                    e = d;
                    d = p / q;
                } else {
                    d = xm; e = d;
                }
            } else {
                d = xm; e = d;
            }
            xa = xb; fa = fb;
            xb += std::fabs(d) > tol1 ? d : (xm > 0 ? tol1 : -tol1);
            F_of(xb, &fb);
        }
        amin_ = xb;
    } else {
        // bracket a minimum of F by golden steps, then Brent's minimiser
        double fa0 = F_of(a0, nullptr);
        double a1 = a0 + h, fa1 = F_of(a1, nullptr);
        if (fa1 > fa0) { std::swap(a0, a1); std::swap(fa0, fa1); }
        double a2 = a1 + GOLD * (a1 - a0), fa2 = F_of(a2, nullptr);
        while (fa1 > fa2) {
            if (nsolve_ >= max_solves) throw std::runtime_error("BRENT: no minimum of F was bracketed");
            a0 = a1; fa0 = fa1; a1 = a2; fa1 = fa2;
            a2 = a1 + GOLD * (a1 - a0);
            if (a2 <= 0) throw std::runtime_error("BRENT: the bracket left the positive cell lengths");
            fa2 = F_of(a2, nullptr);
        }
        double lo_a = std::min(a0, a2), hi_a = std::max(a0, a2);
        double x = a1, w = a1, v = a1, fx = fa1, fw = fa1, fv = fa1, d = 0.0, e = 0.0;
        while (nsolve_ < max_solves) {
            const double xm = 0.5 * (lo_a + hi_a);
            const double tol1 = tol * std::fabs(x) + 1e-20, tol2 = 2.0 * tol1;
            if (std::fabs(x - xm) <= tol2 - 0.5 * (hi_a - lo_a)) break;
            bool golden = true;
            if (std::fabs(e) > tol1) {
                double r = (x - w) * (fx - fv), q = (x - v) * (fx - fw), p = (x - v) * q - (x - w) * r;
                q = 2.0 * (q - r);
                if (q > 0) p = -p;
                q = std::fabs(q);
                const double eprev = e;
                e = d;
                if (std::fabs(p) < std::fabs(0.5 * q * eprev) && p > q * (lo_a - x) && p < q * (hi_a - x)) {
                    d = p / q;
                    const double u = x + d;
                    if (u - lo_a < tol2 || hi_a - u < tol2) d = xm > x ? tol1 : -tol1;
                    golden = false;
                }
            }
            if (golden) {
                e = x >= xm ? lo_a - x : hi_a - x;
                d = CGOLD * e;
            }
            const double u = std::fabs(d) >= tol1 ? x + d : x + (d > 0 ? tol1 : -tol1);
            const double fu = F_of(u, nullptr);
            if (fu <= fx) {
                (u >= x ? lo_a : hi_a) = x;
                v = w; fv = fw; w = x; fw = fx; x = u; fx = fu;
            } else {
                (u < x ? lo_a : hi_a) = u;
                if (fu <= fw || w == x) { v = w; fv = fw; w = u; fw = fu; }
                else if (fu <= fv || v == x || v == w) { v = u; fv = fu; }
            }
        }
        amin_ = x;
    }
    // leave the model at the optimum (the last solve may have been elsewhere)
    const std::vector<double>& last = trace_.back();
    double b, c;
    update_cell(amin_, b, c);
    if (std::fabs(last[0] - amin_) > 0.0) solve_cell(amin_, nullptr);
    Fmin_ = Hlast_;
    std::vector<double> l = m->lengths();
    std::cout << "amin = " << std::setprecision(10) << l[0] << " bmin = " << l[1] << " cmin = " << l[2] << "\n"
              << "Fmin = " << std::setprecision(15) << Fmin_ << std::setprecision(6) << "\n";
}

void scft::save_cell(const std::string& file) const {
    const int n = (int)trace_.size();
    std::vector<double> as(n), bs(n), cs(n), Fs(n);
    for (int i = 0; i < n; i++) {
        as[i] = trace_[i][0]; bs[i] = trace_[i][1]; cs[i] = trace_[i][2]; Fs[i] = trace_[i][3];
    }
    std::map<std::string, std::pair<std::vector<int>, std::vector<double>>> vars;
    vars["a"] = {{n, 1}, as};
    vars["b"] = {{n, 1}, bs};
    vars["c"] = {{n, 1}, cs};
    vars["F"] = {{n, 1}, Fs};
    mat_write(file, vars);
}

// scft::relax (src/scft.cc:382-422) with save_data's stop tests
// (:532-587): non-finite H stops (diverged); residual below thresh_residual
// after min_iter stops (converged); max_iter stops.  Updates between record
// points run as one batch of graph replays.
void scft::relax() {
    const int max_iter = cfg_.max_iter();
    const int rec = std::max(1, cfg_.record_interval());
    const bool save = cfg_.is_save_data();
    int i = 0;
    while (i < max_iter) {
        int n = save ? std::min(rec - (i % rec), max_iter - i) : max_iter - i;
        static_cast<Model_AB*>(m_)->update(n);
        i += n;
        iter_ = i;
        if (cfg_.is_display() && cfg_.display_interval() > 0 && i % cfg_.display_interval() == 0) {
            std::cout << i << "\n";
            m_->display();
        }
        if (save && i % rec == 0) {
            Hlast_ = m_->H();
            rlast_ = m_->residual_error();
            if (!std::isfinite(Hlast_)) {
                std::cout << "\nError: diverge\nIter: " << i << "\nH = " << Hlast_ << "\n";
                return;
            }
            if (i > cfg_.min_iter() && i / rec > 1 && rlast_ < cfg_.thresh_residual()) break;
        }
    }
    Hlast_ = m_->H();
    rlast_ = m_->residual_error();
}

}  // namespace polyorder
