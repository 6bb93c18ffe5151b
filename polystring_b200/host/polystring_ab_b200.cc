// polystring_ab_b200.cc -- the string-method application of the reference
// (scft/polystring_AB.cc:70-329) on the B200 backend.
//
//   polystring_ab_b200 [paramString.ini]
//
// Reads the reference's string config unchanged ([string] num_of_beads,
// string_iteration, save_string_interval, thresh_string_H, is_readString,
// is_changeSize, and the model / grid / MDE / SCFT sections), builds the
// initial string from the end states in defect.mat and vLam.mat (or reads a
// whole string from stringData.mat), then runs string iterations until
//
//   max over images |H(st) - H(st-1)| <= thresh_string_H  or  st == string_iteration
//
// (polystring_AB.cc:125-150).  One string iteration (the SCFT of every image,
// arc length, spline re-sampling, ends restored) is one ps_string_ab_iterate
// call.  Every save_string_interval iterations, and once more at the end,
// result.mat gets wa, wb, phia, phib (m x Lx x Ly x Lz) and the F, H, S, dH
// records (save_data, polystring_AB.cc:226-254).  Files are read and written
// next to the config file.
//
// Not provided: is_changeSize = true (a cell size per image); the device
// string runs one cell for all images, and the run stops with an error.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "polyorder.h"
#include "polystring_b200.h"

namespace {

using polyorder::Config;

void check(int rc) {
    if (rc != PS_OK) throw std::runtime_error(ps_last_error());
}

// one field of a MAT-file, 3D (Lx, Ly, Lz) column-major -> row-major (z fastest)
std::vector<double> read3(const std::string& file, const std::string& name, int Lx, int Ly, int Lz) {
    polyorder::Grid g(Lx, Ly, Lz);
    g.load_mat(file, name);
    return g.vec();
}

// a whole string, 4D (m, Lx, Ly, Lz) column-major (input_data4,
// polystring_AB.cc:169-182) -> image-major row-major
std::vector<double> read4(const std::string& file, const std::string& name, int m, int Lx, int Ly, int Lz) {
    std::vector<int> dims;
    std::vector<double> v = polyorder::mat_read(file, name, &dims);
    const size_t M = (size_t)Lx * Ly * Lz;
    if (v.size() != (size_t)m * M) throw std::runtime_error("size of " + name + " in " + file + " does not match the string");
    std::vector<double> out(v.size());
    for (int s = 0; s < m; s++)
        for (int i = 0; i < Lx; i++)
            for (int j = 0; j < Ly; j++)
                for (int k = 0; k < Lz; k++)
                    out[s * M + ((size_t)i * Ly + j) * Lz + k] = v[s + (size_t)m * (i + (size_t)Lx * (j + (size_t)Ly * k))];
    return out;
}

// image-major row-major -> (m, Lx, Ly, Lz) column-major
std::vector<double> to4(const std::vector<double>& a, int m, int Lx, int Ly, int Lz) {
    const size_t M = (size_t)Lx * Ly * Lz;
    std::vector<double> out(a.size());
    for (int s = 0; s < m; s++)
        for (int i = 0; i < Lx; i++)
            for (int j = 0; j < Ly; j++)
                for (int k = 0; k < Lz; k++)
                    out[s + (size_t)m * (i + (size_t)Lx * (j + (size_t)Ly * k))] = a[s * M + ((size_t)i * Ly + j) * Lz + k];
    return out;
}

// (rows, cols) row-major record -> column-major
std::vector<double> to2(const std::vector<double>& a, int rows, int cols) {
    std::vector<double> out(a.size());
    for (int r = 0; r < rows; r++)
        for (int c = 0; c < cols; c++) out[r + (size_t)rows * c] = a[(size_t)r * cols + c];
    return out;
}

}  // namespace

int main(int argc, char** argv) {
    const std::string file = argc > 1 ? argv[1] : "paramString.ini";
    try {
        Config cfg(file);
        const int m = cfg.get_integer("string", "num_of_beads");
        const int maxT = cfg.get_integer("string", "string_iteration");
        const int save_interval = std::max(1, cfg.get_integer("string", "save_string_interval", 1));
        const bool read_string = cfg.get_bool("string", "is_readString");
        const bool change_size = cfg.get_bool("string", "is_changeSize");
        const double thresh = cfg.get_double("string", "thresh_string_H");
        if (change_size)
            throw std::runtime_error("is_changeSize = true (a cell size per image) is not provided by the B200 backend");
        if (m < 3 || maxT < 1) throw std::runtime_error("[string] needs num_of_beads >= 3 and string_iteration >= 1");
        const int Lx = cfg.Lx(), Ly = cfg.Ly(), Lz = cfg.Lz();
        const size_t M = (size_t)Lx * Ly * Lz;

        ps_model_ab_params p{};
        p.dim = cfg.dim();
        p.Lx = Lx; p.Ly = Ly; p.Lz = Lz;
        p.cell = polyorder::UnitCell(cfg).c_cell();
        std::vector<double> Ms = cfg.Ms(), lam = cfg.lam();
        p.sA = (int)Ms.at(0);
        p.sB = (int)Ms.at(1);
        p.chiN = cfg.chiN();
        p.lamA = lam.at(0); p.lamB = lam.at(1); p.lamYita = lam.at(2);
        p.mde = cfg.algo_mde_type() == polyorder::AlgorithmMDEType::OS2 ? PS_MDE_OS2 : PS_MDE_RQM4;
        if (cfg.algo_mde_type() == polyorder::AlgorithmMDEType::ETDRK4)
            throw std::runtime_error("ETDRK4 is not provided by the B200 backend (RQM4, OS2)");
        p.scft = PS_SCFT_EM;   // images restart from DATA_INIT fields with simple mixing (resetInString)
        p.n_anderson = 1;
        p.compressible = cfg.is_compressible() ? 1 : 0;
        p.contour = cfg.algo_contour_integration_type() == polyorder::AlgorithmContourType::TRAPEZOIDAL
                        ? PS_CONTOUR_TRAPEZOID : PS_CONTOUR_SIMPSON;

        // ---- initial string (initialize_string, polystring_AB.cc:184-224) ------
        const std::string dir = cfg.dir();
        std::vector<double> wa(m * M), wb(m * M), phia(m * M), phib(m * M);
        if (read_string) {
            std::printf("Initialization from an existing string!\n");
            wa = read4(dir + "stringData.mat", "wa", m, Lx, Ly, Lz);
            wb = read4(dir + "stringData.mat", "wb", m, Lx, Ly, Lz);
            phia = read4(dir + "stringData.mat", "phia", m, Lx, Ly, Lz);
            phib = read4(dir + "stringData.mat", "phib", m, Lx, Ly, Lz);
        } else {
            std::printf("Initializing string by two ends!\n");
            const char* names[4] = {"wA", "wB", "phiA", "phiB"};
            std::vector<double>* dst[4] = {&wa, &wb, &phia, &phib};
            for (int f = 0; f < 4; f++) {
                std::vector<double> e0 = read3(dir + "defect.mat", names[f], Lx, Ly, Lz);
                std::vector<double> e1 = read3(dir + "vLam.mat", names[f], Lx, Ly, Lz);
                for (int i = 0; i < m; i++)
                    for (size_t g = 0; g < M; g++)
                        (*dst[f])[i * M + g] = e0[g] + 1.0 * i / (m - 1) * (e1[g] - e0[g]);
            }
        }
        std::fflush(stdout);
        // the ends' densities, restored into every saved string (redistribute_stringBeads :321-328)
        std::vector<double> phiae(phia.begin(), phia.begin() + M), phibe(phib.begin(), phib.begin() + M);
        std::vector<double> phiae1(phia.end() - M, phia.end()), phibe1(phib.end() - M, phib.end());

        ps_string_ab* st_h = nullptr;
        check(ps_string_ab_create(&p, m, cfg.max_iter(), &st_h));
        check(ps_string_ab_set_images(st_h, wa.data(), wb.data()));

        std::vector<double> H((size_t)maxT * m, 0.0), S((size_t)maxT * m, 0.0), dH((size_t)maxT * m, 10.0);
        std::vector<double> F(maxT, 0.0);
        auto save_data = [&]() {
            check(ps_string_ab_get(st_h, 0, wa.data()));
            check(ps_string_ab_get(st_h, 1, wb.data()));
            check(ps_string_ab_get(st_h, 2, phia.data()));
            check(ps_string_ab_get(st_h, 3, phib.data()));
            std::copy(phiae.begin(), phiae.end(), phia.begin());
            std::copy(phibe.begin(), phibe.end(), phib.begin());
            std::copy(phiae1.begin(), phiae1.end(), phia.end() - M);
            std::copy(phibe1.begin(), phibe1.end(), phib.end() - M);
            std::vector<int> d4 = {m, Lx, Ly, Lz}, d1 = {maxT}, d2 = {maxT, m};
            polyorder::mat_write(dir + "result.mat",
                                 {{"wa", {d4, to4(wa, m, Lx, Ly, Lz)}},
                                  {"wb", {d4, to4(wb, m, Lx, Ly, Lz)}},
                                  {"phia", {d4, to4(phia, m, Lx, Ly, Lz)}},
                                  {"phib", {d4, to4(phib, m, Lx, Ly, Lz)}},
                                  {"F", {d1, F}},
                                  {"H", {d2, to2(H, maxT, m)}},
                                  {"S", {d2, to2(S, maxT, m)}},
                                  {"dH", {d2, to2(dH, maxT, m)}}});
        };

        // ---- string iterations (run_string, polystring_AB.cc:111-152) -----------
        auto t0 = std::chrono::steady_clock::now();
        int st = 0;
        double maxdH = 0.0;
        do {
            check(ps_string_ab_iterate(st_h, 1));
            double* h = H.data() + (size_t)st * m;
            check(ps_string_ab_H(st_h, h));
            check(ps_string_ab_S(st_h, S.data() + (size_t)st * m));
            double f = 0.0;
            for (int s = 0; s < m; s++) f += h[s];
            F[st] = f / m;
            if (st > 0)
                for (int s = 0; s < m; s++) dH[(size_t)st * m + s] = std::fabs(h[s] - h[s - m]);
            maxdH = *std::max_element(dH.begin() + (size_t)st * m, dH.begin() + (size_t)(st + 1) * m);
            std::printf("string iteration %d: F = %.15f, max dH = %.6e\n", st, F[st], maxdH);
            if (st % save_interval == 0) save_data();
            st += 1;
        } while (maxdH > thresh && st < maxT);
        save_data();
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("string iterations = %d\n", st);
        std::printf("F = %.15f\n", F[st - 1]);
        std::printf("The whole time is %g\n", secs);
        ps_string_ab_destroy(st_h);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
}
