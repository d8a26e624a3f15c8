// cabi_adapter.cpp -- a C++ translation unit that drives libmphy.so through the SolverGpu adapter
// (include/mphy_solver_gpu.hpp) the way femSolidmechanics drives SolverPetsc. Built and run by
// tests/test_cabi_cpp.py: compiled with g++ against include/ on the CPU (syntax and link), run on
// the GPU against the oracle.
//
//   cabi_adapter <input.bin> <output.bin>
//
// input.bin (little-endian): int32 n_node, n_elem, npe, n_mat, n_free; f64 coords[3 n_node];
// i32 conn[n_elem npe]; i32 mat_id[n_elem]; f64 mats[3 n_mat]; u8 fixed[3 n_node];
// f64 fnodal[3 n_node]; f64 lambda; i32 row_nnz[n_free] (the reference's d_nnz);
// i32 forAssyVec[n_elem][3 npe]; f64 Ke[n_elem][3 npe][3 npe] (row-major); f64 Fe[n_elem][3 npe].
// output.bin: f64 du_fused[3 n_node]; f64 du_elem[3 n_node]; f64 norm_fused, norm_elem;
// i32 its_fused, its_elem, status_before_assembly.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "mphy_solver_gpu.hpp"

namespace {

// Column-major dense matrix and vector with Eigen's (i, j) / (i) access, standing in for the
// MatrixXd / VectorXd that the reference's element loop hands to assembleMatrixAndVector.
struct ColMat {
    int n = 0;
    std::vector<double> a;
    explicit ColMat(int size) : n(size), a((size_t)size * size) {}
    double& operator()(int i, int j) { return a[(size_t)j * n + i]; }
};
struct Vec {
    std::vector<double> a;
    explicit Vec(int size) : a(size) {}
    double& operator()(int i) { return a[i]; }
};

template <class T>
void read(FILE* f, T* p, size_t n) {
    if (n && fread(p, sizeof(T), n, f) != n) throw std::runtime_error("short input file");
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 2;
    }
    try {
        FILE* f = fopen(argv[1], "rb");
        if (!f) throw std::runtime_error("cannot open input");
        int32_t hdr[5];
        read(f, hdr, 5);
        const int n_node = hdr[0], n_elem = hdr[1], npe = hdr[2], n_mat = hdr[3], n_free = hdr[4];
        const int ns = 3 * npe;
        std::vector<double> coords(3 * (size_t)n_node), mats(3 * (size_t)n_mat), fnodal(3 * (size_t)n_node);
        std::vector<int32_t> conn((size_t)n_elem * npe), mat_id(n_elem), row_nnz(n_free),
            for_assy((size_t)n_elem * ns);
        std::vector<unsigned char> fixed(3 * (size_t)n_node);
        std::vector<double> Ke((size_t)n_elem * ns * ns), Fe((size_t)n_elem * ns);
        double lambda = 0.0;
        read(f, coords.data(), coords.size());
        read(f, conn.data(), conn.size());
        read(f, mat_id.data(), mat_id.size());
        read(f, mats.data(), mats.size());
        read(f, fixed.data(), fixed.size());
        read(f, fnodal.data(), fnodal.size());
        read(f, &lambda, 1);
        read(f, row_nnz.data(), row_nnz.size());
        read(f, for_assy.data(), for_assy.size());
        read(f, Ke.data(), Ke.size());
        read(f, Fe.data(), Fe.size());
        fclose(f);

        // setSolver(SOLVER_LIB_PETSC) -> prepareMatrixPattern -> initialise(n, n, d_nnz, o_nnz)
        SolverGpu slv;
        slv.opts.rtol = 1e-12;
        slv.setMesh(n_node, coords.data(), n_elem, npe, conn.data(), mat_id.data(), n_mat, mats.data(),
                    fixed.data());
        std::vector<int> offdiag(n_free, 0);
        slv.initialise(n_free, n_free, row_nnz.data(), offdiag.data());
        slv.Fext = fnodal;
        for (size_t i = 0; i < for_assy.size(); ++i)
            if (slv.forAssyVec()[i] != for_assy[i]) throw std::runtime_error("forAssyVec differs from the input's");
        const int32_t status_before = slv.factoriseAndSolve();  // -1: not assembled yet

        // (1) the fused GPU path: one Newton iteration from u = 0 on host displacements
        std::vector<double> du_fused(3 * (size_t)n_node, 0.0);
        const double norm_fused = slv.newtonIteration(du_fused, lambda);
        const int32_t its_fused = slv.last_its;

        // (2) the reference's element loop: Klocal / Flocal per element, assembled through
        // assembleMatrixAndVector(0, 0, forAssyVec, forAssyVec, Klocal, Flocal), in descending
        // element order to show the order does not matter
        slv.zeroMtx();
        ColMat K(ns);
        Vec F(ns);
        std::vector<int> row(ns);
        for (int e = n_elem - 1; e >= 0; --e) {
            for (int i = 0; i < ns; ++i) {
                row[i] = for_assy[(size_t)e * ns + i];
                F(i) = Fe[(size_t)e * ns + i];
                for (int j = 0; j < ns; ++j) K(i, j) = Ke[((size_t)e * ns + i) * ns + j];
            }
            slv.assembleMatrixAndVector(0, 0, row, row, K, F);
        }
        slv.addExternalForces(lambda);
        const double norm_elem = slv.rhsNorm();
        if (slv.factoriseAndSolve() != 0) throw std::runtime_error("factoriseAndSolve failed");
        const int32_t its_elem = slv.last_its;
        std::vector<double> du_elem;
        slv.getSolution(du_elem);

        FILE* o = fopen(argv[2], "wb");
        if (!o) throw std::runtime_error("cannot open output");
        fwrite(du_fused.data(), sizeof(double), du_fused.size(), o);
        fwrite(du_elem.data(), sizeof(double), du_elem.size(), o);
        fwrite(&norm_fused, sizeof(double), 1, o);
        fwrite(&norm_elem, sizeof(double), 1, o);
        fwrite(&its_fused, sizeof(int32_t), 1, o);
        fwrite(&its_elem, sizeof(int32_t), 1, o);
        fwrite(&status_before, sizeof(int32_t), 1, o);
        fclose(o);
        printf("adapter ok: n_free=%d its_fused=%d its_elem=%d\n", n_free, its_fused, its_elem);
        return 0;
    } catch (const std::exception& ex) {
        fprintf(stderr, "cabi_adapter: %s\n", ex.what());
        return 1;
    }
}
