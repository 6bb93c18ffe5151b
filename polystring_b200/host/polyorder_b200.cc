// polyorder_b200.cc -- the plain-SCFT application (scft/polyorder.cc:39-115)
// on the B200 backend: reads the reference's param.ini, builds Model_AB,
// runs scft and prints the final free energy.
//
//   polyorder_b200 [param.ini]
//   polyorder_b200 --check param.ini   (parse only: print the model parameters)
//   polyorder_b200 --mat file.mat name (print one variable of a MAT-file)
#include <chrono>
#include <cstdio>
#include <iostream>

#include "polyorder.h"

static void print_params(const polyorder::Config& cfg) {
    polyorder::UnitCell uc(cfg);
    const ps_unit_cell& c = uc.c_cell();
    std::vector<double> Ms = cfg.Ms(), lam = cfg.lam();
    std::printf("dim %d grid %d %d %d\n", cfg.dim(), cfg.Lx(), cfg.Ly(), cfg.Lz());
    std::printf("cell system %d a %.17g b %.17g c %.17g\n", c.system, c.a, c.b, c.c);
    std::printf("Ms %d %d chiN %.17g\n", (int)Ms.at(0), (int)Ms.at(1), cfg.chiN());
    std::printf("lam %.17g %.17g %.17g\n", lam.at(0), lam.at(1), lam.at(2));
    std::printf("mde %d scft %d contour %d cellopt %d init %d etdrk4_M %d\n", (int)cfg.algo_mde_type(),
                (int)cfg.algo_scft_type(), (int)cfg.algo_contour_integration_type(),
                (int)cfg.algo_cell_optimization_type(), (int)cfg.get_grid_init_type(), cfg.etdrk4_M());
    std::printf("n_anderson %d compressible %d max_iter %d min_iter %d record %d thresh %.17g\n",
                cfg.n_Anderson_mixing(), (int)cfg.is_compressible(), cfg.max_iter(), cfg.min_iter(),
                cfg.record_interval(), cfg.thresh_residual());
    std::printf("field_data %s\n", cfg.field_data_file().c_str());
    if (cfg.get_grid_init_type() == polyorder::GridInitType::FILE_INIT) {
        std::string f = cfg.field_data_file();
        if (!f.empty() && f[0] != '/') f = cfg.dir() + f;
        for (const char* name : {"wA", "wB"}) {
            polyorder::Grid g(cfg.Lx(), cfg.Ly(), cfg.Lz());
            g.load_mat(f, name);
            std::printf("%s mean %.17g first %.17g last %.17g\n", name, g.quadrature(), g.data()[0],
                        g.data()[g.size() - 1]);
        }
    }
}

// --mat file name: the variable as the MAT-v5 reader returns it (dims, then
// every value in file order, %.17g)
static int print_mat(const std::string& file, const std::string& name) {
    std::vector<int> dims;
    std::vector<double> v = polyorder::mat_read(file, name, &dims);
    std::printf("dims");
    for (int d : dims) std::printf(" %d", d);
    std::printf("\nvalues");
    for (double x : v) std::printf(" %.17g", x);
    std::printf("\n");
    return 0;
}

int main(int argc, char** argv) {
    if (argc > 3 && std::string(argv[1]) == "--mat") {
        try {
            return print_mat(argv[2], argv[3]);
        } catch (const std::exception& e) {
            std::cerr << "error: " << e.what() << "\n";
            return 1;
        }
    }
    const bool check_only = argc > 1 && std::string(argv[1]) == "--check";
    const std::string file = argc > (check_only ? 2 : 1) ? argv[check_only ? 2 : 1] : "param.ini";
    try {
        polyorder::Config cfg(file);
        if (check_only) {
            print_params(cfg);
            return 0;
        }
        std::string model = cfg.get_string("Model", "model", "AB");
        for (auto& ch : model) ch = (char)toupper((unsigned char)ch);
        if (model != "AB") {
            std::cerr << "model " << model << " is not provided by the B200 backend (AB)\n";
            return 1;
        }
        auto t0 = std::chrono::steady_clock::now();
        polyorder::Model_AB m(cfg);
        polyorder::scft sim(cfg, &m);
        sim.run();
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (cfg.is_save_data()) {
            m.save(cfg.dir() + cfg.base_dir() + cfg.data_file() + ".mat");
            if (!sim.cell_trace().empty()) sim.save_cell(cfg.dir() + cfg.base_dir() + cfg.data_file() + "_cell.mat");
        }
        std::printf("iterations = %d\n", sim.iterations());
        std::printf("residual = %.6e\n", sim.final_residual());
        std::printf("H = %.15f\n", sim.final_H());
        std::printf("Total time elapsed in second:\t%g\n", secs);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
}
