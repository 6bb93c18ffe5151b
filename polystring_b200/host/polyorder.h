// polyorder.h -- C++ host classes with the names and call shapes of
// PolyOrder's SCFT path, running on the B200 through the C ABI of
// include/polystring_b200.h.
//
// The reference's interface types (blitz::Array, arma::vec) are replaced by
// plain contiguous FP64 storage (row-major (x, y, z), z fastest); the class
// and method names, their argument meaning and the config file stay those of
// the reference:
//
//   Config          include/Config.h:51-305 (INI sections and keys)
//   UnitCell        include/UnitCell.h:39-98
//   Grid            include/Grid.h:61-183 (quadrature = mean on a regular grid)
//   Updater         include/Updater.h:44-69 (propagator / density solve, clone)
//   RQM4            include/RQM4.h:44-45, src/RQM4.cc
//   PseudoSpectral  include/PseudoSpectral.h:53-55, src/PseudoSpectral.cc
//   Propagator      include/Propagator.h:40-91
//   Density         include/Density.h:40-88, Simpson (src/Simpson.cc),
//                   Quad4_Closed (src/Quadrature4.cc)
//   Model, Model_AB include/Model.h:46-87, include/Model_AB.h:48-114
//   scft            include/scft.h:56-109 (relax loop, record/convergence; SINGLE,
//                   MANUAL and BRENT cell runs, scft.cc:40-309)
//
// Errors from the device are reported by throwing std::runtime_error with
// the library's message (the reference calls exit(1) on configuration errors).
#pragma once

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "polystring_b200.h"

namespace polyorder {

// ---------------------------------------------------------------------------
// Config: INI file with the reference's sections and keys
// ---------------------------------------------------------------------------
enum class AlgorithmMDEType { OS2, RQM4, ETDRK4 };
enum class AlgorithmSCFTType { EM, ANDERSON };
enum class AlgorithmContourType { TRAPEZOIDAL, SIMPSON };
enum class AlgorithmCellType { SINGLE, BRENT, MANUAL };
enum class GridInitType { RANDOM_INIT, CONSTANT_INIT, FILE_INIT, DATA_INIT, PATTERN_INIT };

class Config {
public:
    explicit Config(const std::string& file);
    std::string get_string(const std::string& section, const std::string& key, const std::string& def = "") const;
    double get_double(const std::string& section, const std::string& key, double def = 0.0) const;
    int get_integer(const std::string& section, const std::string& key, int def = 0) const;
    bool get_bool(const std::string& section, const std::string& key, bool def = false) const;
    std::vector<double> get_list(const std::string& section, const std::string& key) const;

    int dim() const { return get_integer("Grid", "dimension", 3); }
    int Lx() const { return get_integer("Grid", "Lx", 1); }
    int Ly() const { return get_integer("Grid", "Ly", 1); }
    int Lz() const { return get_integer("Grid", "Lz", 1); }
    double a() const { return get_double("UnitCell", "a"); }
    double b() const { return get_double("UnitCell", "b"); }
    double c() const { return get_double("UnitCell", "c"); }
    void a(double v) { set("UnitCell", "a", v); }
    void b(double v) { set("UnitCell", "b", v); }
    void c(double v) { set("UnitCell", "c", v); }
    std::string crystal_system() const { return get_string("UnitCell", "CrystalSystemType"); }
    std::vector<double> Ms() const { return get_list("Algorithm_MDE", "Ms"); }
    double chiN() const { return get_list("Model", "chiN").at(0); }
    std::vector<double> lam() const { return get_list("Algorithm_SCFT", "lam"); }
    bool is_compressible() const { return get_bool("Model", "is_compressible"); }
    int n_Anderson_mixing() const { return get_integer("Algorithm_SCFT", "n_Anderson_mixing", 5); }
    // Config::etdrk4_M (Config.cc:1203-1205); empty or <= 0: Etdrk4_PBC's default
    int etdrk4_M() const { return get_integer("Algorithm_MDE", "etdrk4_M", 0); }
    int min_iter() const { return get_integer("Algorithm_SCFT", "min_iter", 1); }
    int max_iter() const { return get_integer("Algorithm_SCFT", "max_iter", 1); }
    double thresh_residual() const { return get_double("Algorithm_SCFT", "thresh_residual", 0.0); }
    int record_interval() const { return get_integer("IO", "record_interval", 1); }
    int display_interval() const { return get_integer("IO", "display_interval", 1); }
    bool is_display() const { return get_bool("IO", "is_display"); }
    bool is_save_data() const { return get_bool("IO", "is_save_data"); }
    std::string base_dir() const { return get_string("IO", "base_dir", "./"); }
    std::string data_file() const { return get_string("IO", "data_file", "scft_out"); }
    std::string field_data_file() const { return get_string("Grid", "field_data"); }
    int seed() const { return get_integer("Grid", "random_seed", 0); }
    AlgorithmMDEType algo_mde_type() const;
    AlgorithmSCFTType algo_scft_type() const;
    AlgorithmContourType algo_contour_integration_type() const;
    AlgorithmCellType algo_cell_optimization_type() const;
    GridInitType get_grid_init_type() const;
    std::string dir() const { return dir_; }

private:
    void set(const std::string& section, const std::string& key, double v);
    std::map<std::string, std::map<std::string, std::string>> kv_;
    std::string dir_;
};

// ---------------------------------------------------------------------------
// UnitCell / Grid
// ---------------------------------------------------------------------------
class UnitCell {
public:
    explicit UnitCell(const Config& cfg);
    const ps_unit_cell& c_cell() const { return cell_; }
    double lx() const { return cell_.a; }
    double ly() const { return cell_.b; }
    double lz() const { return cell_.c; }

private:
    ps_unit_cell cell_;
};

class Grid {
public:
    Grid() = default;
    Grid(int Lx, int Ly, int Lz, double val = 0.0) : Lx_(Lx), Ly_(Ly), Lz_(Lz), data_((size_t)Lx * Ly * Lz, val) {}
    int Lx() const { return Lx_; }
    int Ly() const { return Ly_; }
    int Lz() const { return Lz_; }
    long size() const { return (long)data_.size(); }
    double* data() { return data_.data(); }
    const double* data() const { return data_.data(); }
    std::vector<double>& vec() { return data_; }
    // Grid::quadrature on a regular grid: the mean (src/Grid.cc:329-374)
    double quadrature() const;
    // read the variable `name` of a MAT-file (Grid::set_value(file), src/Grid.cc:694-711)
    void load_mat(const std::string& file, const std::string& name);

private:
    int Lx_ = 1, Ly_ = 1, Lz_ = 1;
    std::vector<double> data_;
};

// MAT-file v5 (uncompressed) double arrays, column-major as MATLAB stores them
std::vector<double> mat_read(const std::string& file, const std::string& name, std::vector<int>* dims = nullptr);
void mat_write(const std::string& file, const std::map<std::string, std::pair<std::vector<int>, std::vector<double>>>& vars);

// ---------------------------------------------------------------------------
// Updaters and propagators
// ---------------------------------------------------------------------------
class Propagator;

class Updater {
public:
    virtual ~Updater() = default;
    // for Propagator (Updater.h:55)
    virtual void solve(Propagator& q, const Grid& w) { (void)q; (void)w; }
    // for Density (Updater.h:57-58)
    virtual void solve(std::vector<double>& data, const Propagator& q, const Propagator& qc, double cc) const {
        (void)data; (void)q; (void)qc; (void)cc;
    }
    virtual Updater* clone() const = 0;
};

class PropagatorUpdater : public Updater {
public:
    PropagatorUpdater(int scheme, const UnitCell& uc, int Lx, int Ly, int Lz, double ds);
    PropagatorUpdater(const PropagatorUpdater& rhs);
    ~PropagatorUpdater() override;
    void solve(Propagator& q, const Grid& w) override;

protected:
    ps_updater* h_ = nullptr;
};

class RQM4 : public PropagatorUpdater {
public:
    RQM4(const UnitCell& uc, int Lx, int Ly, int Lz, double ds) : PropagatorUpdater(PS_MDE_RQM4, uc, Lx, Ly, Lz, ds) {}
    RQM4* clone() const override { return new RQM4(*this); }
};

class PseudoSpectral : public PropagatorUpdater {
public:
    PseudoSpectral(const UnitCell& uc, int Lx, int Ly, int Lz, double ds)
        : PropagatorUpdater(PS_MDE_OS2, uc, Lx, Ly, Lz, ds) {}
    PseudoSpectral* clone() const override { return new PseudoSpectral(*this); }
};

class Propagator : public Grid {
public:
    Propagator(int len, double ds, int Lx, int Ly, int Lz, Updater* up = nullptr)
        : Grid(Lx, Ly, Lz), len_(len), ds_(ds), qs_((size_t)len * Lx * Ly * Lz, 0.0), up_(up) {}
    int len() const { return len_; }
    double ds() const { return ds_; }
    double* qs() { return qs_.data(); }
    const double* qs() const { return qs_.data(); }
    void set_head(const double* u);
    const double* get_tail() const { return qs_.data() + (size_t)(len_ - 1) * size(); }
    void update(const Grid& w) { up_->solve(*this, w); }
    double Q(int s) const;
    double Qt() const { return Q(len_ - 1); }

private:
    int len_;
    double ds_;
    std::vector<double> qs_;
    Updater* up_;
};

class DensityUpdater : public Updater {
public:
    explicit DensityUpdater(int rule) : rule_(rule) {}
    void solve(std::vector<double>& data, const Propagator& q, const Propagator& qc, double cc) const override;

private:
    int rule_;
};
class Simpson : public DensityUpdater {
public:
    Simpson() : DensityUpdater(PS_CONTOUR_SIMPSON) {}
    Simpson* clone() const override { return new Simpson(*this); }
};
class Quad4_Closed : public DensityUpdater {
public:
    Quad4_Closed() : DensityUpdater(PS_CONTOUR_QUAD4_CLOSED) {}
    Quad4_Closed* clone() const override { return new Quad4_Closed(*this); }
};

class Density : public Grid {
public:
    Density(int Lx, int Ly, int Lz, const Updater* up = nullptr)
        : Grid(Lx, Ly, Lz), up_(up ? up->clone() : nullptr) {}
    ~Density() { delete up_; }
    void update(const Propagator& q, const Propagator& qc, double cc);

private:
    Updater* up_;
};

// ---------------------------------------------------------------------------
// Model / Model_AB / scft
// ---------------------------------------------------------------------------
class Model {
public:
    virtual ~Model() = default;
    virtual void update() = 0;
    virtual double H() const = 0;
    virtual double Hw() const = 0;
    virtual double Hs() const = 0;
    virtual double residual_error() const = 0;
    virtual void display() const = 0;
    virtual void save(const std::string& file) = 0;
};

class Model_AB : public Model {
public:
    explicit Model_AB(const Config& cfg);
    ~Model_AB() override;
    void update() override;                 // Model_AB::update (src/Model_AB.cc:136-261)
    void update(int n);                     // n updates in one call (graph replays)
    double H() const override;
    double Hw() const override;
    double Hs() const override;
    double residual_error() const override;
    double Q() const;
    void display() const override;
    void save(const std::string& file) override;
    std::vector<double> field(int which) const;   // PS_FIELD_*
    void set_fields(const std::vector<double>& wA, const std::vector<double>& wB);
    // scft::reset_model with DATA_INIT (scft.cc:362-380, Model_AB.cc:20-28):
    // the same model on the cell of cfg, continuing from the current fields
    void reset_cell(const Config& cfg);
    // the cell lengths (lx, ly, lz) the model runs on
    std::vector<double> lengths() const;
    // d(-ln Q)/dl_i at the current fields (adjoint of the RQM4 chain; 2D/3D)
    bool has_stress() const;
    std::vector<double> stress() const;

private:
    ps_model_ab* h_ = nullptr;
    ps_model_ab_params p_;
    int Lx_, Ly_, Lz_;
};

class scft {
public:
    scft(const Config& cfg, Model* pmodel) : cfg_(cfg), m_(pmodel) {}
    // scft::run (src/scft.cc:40-105): SINGLE relaxes the configured cell;
    // MANUAL relaxes every cell of the batch_cell_min/step/max grid; BRENT
    // finds the cell length a of least free energy (see optimize_cell)
    void run();
    void relax();    // scft::relax (src/scft.cc:382-422)
    int iterations() const { return iter_; }
    double final_H() const { return Hlast_; }
    double final_residual() const { return rlast_; }
    // cells solved so far (lx, ly, lz, F), the as/bs/cs/Fs record of scft.h
    const std::vector<std::vector<double>>& cell_trace() const { return trace_; }
    double amin() const { return amin_; }
    double Fmin() const { return Fmin_; }
    // the cell record as a MAT-file (scft::save_cell, src/scft.cc:589-609)
    void save_cell(const std::string& file) const;

private:
    // scft::update_cell (src/scft.cc:107-121): b and c follow a on regular grids
    void update_cell(double a, double& b, double& c) const;
    // relax on cell a (continuing from the current fields); returns F = H and,
    // when dFda is given, dF/da from the adjoint stress
    double solve_cell(double a, double* dFda);
    void optimize_cell();
    Config cfg_;
    Model* m_;
    int iter_ = 0, nsolve_ = 0;
    double Hlast_ = 0.0, rlast_ = 0.0;
    double amin_ = 0.0, Fmin_ = 0.0;
    std::vector<std::vector<double>> trace_;
};

}  // namespace polyorder
