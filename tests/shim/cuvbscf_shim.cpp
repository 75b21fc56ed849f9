// The reference-side shim a maintainer would add to route the `cuvbscf` method flag to vbcore,
// compiled and run by tests/test_shim.py (test infrastructure: the structs below are minimal
// stand-ins for the reference's types, std::vector instead of Eigen).
//
// It mirrors xmvb::cuda::solve_scf(Context&, const VbScfInput&, AoPairGraph&&, double
// nuclear_repulsion, const VbScfOptimizerOptions&, observe) -> ScfResult (src/cuda/vb/scf.hpp:41-46
// of the reference): the deck's AO integrals (libcint in the reference) arrive as the AoPairGraph's
// unique-integral stream (src/integrals/ao/input.hpp:36-60) and are handed to
// vb_scf_problem_create_from_integrals; the orbital optimization runs in vb_solve_scf.  The host
// ERI payload is consumed (moved in and released after the problem is built), and errors become
// exceptions as in the reference (VB_ERR_INVALID -> std::invalid_argument, others ->
// std::runtime_error).
//
// main() reads one problem from a text file (argv[1]) and prints the result.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "vbcore.h"

namespace shim {

// The AO pair graph's unique-integral stream: AO pairs, then (left pair, right pair, value) with
// each unordered pair of pairs once.
struct AoPairGraph {
    std::vector<int32_t> pair_first, pair_second;
    std::vector<int64_t> integral_rows, integral_columns;
    std::vector<double> integral_values;
};

struct VbScfInput {
    int n_basis = 0;
    std::vector<double> ao_overlap, core_hamiltonian;  // column-major n_bf x n_bf
    std::vector<std::vector<int>> active_fragments;     // basis functions of each active orbital
    int n_electrons = 0, multiplicity = 1;
    std::string structure_class = "COV";
    std::vector<double> initial_orbitals;               // n_bf x n_active, column-major
};

struct VbScfOptimizerOptions {
    int max_iterations = 200;
    double gradient_tolerance = 1e-6;
    int history = 100;
    double armijo = 1e-4;
};

struct ScfResult {
    bool converged = false;
    double energy = 0.0;
    double gradient_inf = 0.0;
    int iterations = 0;
    std::vector<double> orbitals;
};

[[noreturn]] void raise(vb_status st, vb_context* ctx) {
    const std::string msg = std::string("XMVB-CPP error: ") + vb_last_error(ctx);
    if (st == VB_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

ScfResult solve_scf(vb_context* ctx, const VbScfInput& input, AoPairGraph&& graph, double nuclear_repulsion,
                    const VbScfOptimizerOptions& options) {
    AoPairGraph g = std::move(graph);  // consumed, as the reference's solve_scf does
    const int n_act = (int)input.active_fragments.size();
    std::vector<int32_t> off{0}, fn;
    for (const auto& f : input.active_fragments) {
        fn.insert(fn.end(), f.begin(), f.end());
        off.push_back((int32_t)fn.size());
    }
    vb_scf_integral_input in{input.n_basis,
                             input.ao_overlap.data(),
                             input.core_hamiltonian.data(),
                             (int64_t)g.pair_first.size(),
                             g.pair_first.data(),
                             g.pair_second.data(),
                             (int64_t)g.integral_values.size(),
                             g.integral_rows.data(),
                             g.integral_columns.data(),
                             g.integral_values.data(),
                             nuclear_repulsion,
                             n_act,
                             off.data(),
                             fn.data(),
                             input.n_electrons,
                             input.multiplicity,
                             input.structure_class.c_str()};
    vb_scf_problem* prob = nullptr;
    vb_status st = vb_scf_problem_create_from_integrals(ctx, &in, &prob);
    g = AoPairGraph{};  // the host payload is released once the problem holds its factors
    if (st != VB_OK) raise(st, ctx);
    vb_scf_options opt{options.max_iterations, options.gradient_tolerance, options.history, options.armijo};
    vb_scf_result res{};
    ScfResult out;
    out.orbitals.assign(input.initial_orbitals.size(), 0.0);
    st = vb_solve_scf(prob, input.initial_orbitals.data(), &opt, &res, out.orbitals.data());
    vb_scf_problem_destroy(prob);
    if (st != VB_OK) raise(st, ctx);
    out.converged = res.converged != 0;
    out.energy = res.energy;
    out.gradient_inf = res.gradient_inf;
    out.iterations = res.iterations;
    return out;
}

}  // namespace shim

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s problem.txt\n", argv[0]);
        return 2;
    }
    std::ifstream f(argv[1]);
    shim::VbScfInput in;
    shim::AoPairGraph g;
    double enuc = 0.0;
    int n_act = 0;
    long long n_pairs = 0, n_int = 0;
    f >> in.n_basis;
    const int n = in.n_basis;
    in.ao_overlap.resize((size_t)n * n);
    in.core_hamiltonian.resize((size_t)n * n);
    for (auto& x : in.ao_overlap) f >> x;
    for (auto& x : in.core_hamiltonian) f >> x;
    f >> n_pairs;
    g.pair_first.resize(n_pairs);
    g.pair_second.resize(n_pairs);
    for (long long p = 0; p < n_pairs; ++p) f >> g.pair_first[p] >> g.pair_second[p];
    f >> n_int;
    g.integral_rows.resize(n_int);
    g.integral_columns.resize(n_int);
    g.integral_values.resize(n_int);
    for (long long t = 0; t < n_int; ++t) f >> g.integral_rows[t] >> g.integral_columns[t] >> g.integral_values[t];
    f >> enuc >> n_act;
    in.active_fragments.resize(n_act);
    for (auto& frag : in.active_fragments) {
        int cnt = 0;
        f >> cnt;
        frag.resize(cnt);
        for (auto& m : frag) f >> m;
    }
    f >> in.n_electrons >> in.multiplicity >> in.structure_class;
    in.initial_orbitals.resize((size_t)n * n_act);
    for (auto& x : in.initial_orbitals) f >> x;
    if (!f) {
        std::fprintf(stderr, "bad problem file\n");
        return 2;
    }
    vb_context* ctx = nullptr;
    if (vb_context_create(0, 0, &ctx) != VB_OK) {
        std::fprintf(stderr, "XMVB-CPP error: %s\n", vb_last_error(nullptr));
        return 2;
    }
    int rc = 0;
    try {
        shim::VbScfOptimizerOptions opt;
        opt.gradient_tolerance = 1e-7;
        const shim::ScfResult r = shim::solve_scf(ctx, in, std::move(g), enuc, opt);
        std::printf("converged %d\nenergy %.15e\ngradient_inf %.3e\niterations %d\n", r.converged ? 1 : 0, r.energy,
                    r.gradient_inf, r.iterations);
        rc = r.converged ? 0 : 2;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        rc = 2;
    }
    vb_context_destroy(ctx);
    return rc;
}
