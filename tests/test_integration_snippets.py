"""The C++ adapter snippets of INTEGRATION.md compile against include/qz_b200.h.

The snippets are the code a maintainer adds to the reference (Simulation, Beam) under QUARZ_B200. The
reference itself does not build here (it needs Kokkos), so its classes are replaced by stubs that declare
exactly the members the snippets use, with the reference's member names; the snippets are compiled in
order in one translation unit with g++ -fsyntax-only (CUDA runtime header for cudaMalloc / cudaMemcpy,
declarations for the two MPI calls of the multi-rank snippet). This checks the entry points' names,
argument counts and types and the field order of every aggregate the snippets fill (qz_species,
qz_beam_view, qz_box, qz_analytic_beam, qz_plasma_state).
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STUBS = r"""
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "qz_b200.h"

typedef double Real;
typedef int MPI_Comm;
#define MPI_DOUBLE 0
#define MPI_STATUS_IGNORE nullptr
int MPI_Recv(void*, int, int, int, int, MPI_Comm, void*);
int MPI_Send(const void*, int, int, int, int, MPI_Comm);

struct View3D { double* data() const; size_t span() const; };
struct GridD { int M() const; double r(int) const; };
struct Cfg { int modes, picard, ab_order; double delta_min, max_qsa; };
struct Comm { int rank() const; int size() const; };
struct SpeciesRef {
    double q() const; double m() const; int ppc() const; int ntheta() const; int mobile() const;
    double density() const; double rmax() const; double channel_depth() const; double channel_radius() const;
};
struct BeamRef {
    double* host_rows7(); int64_t n() const; double q() const; double m() const; int rigid() const;
    double gref() const; double xiref() const;
};
struct Instance {
    std::vector<double> nodes; qz_sweep_params params; int nbeams; const double* const* rows7;
    const int64_t* n; const double* q; const double* m; const int* rigid; const double* gref; const double* xiref;
};

struct Simulation {
    qz_grid* qz_g_; qz_sweep* qz_s_;
    double *d_bsrc_, *d_fld_, *d_diag_, *d_state_in_, *d_state_out_, *d_guard_;
    GridD grid_; Cfg cfg_; Comm comm_;
    double xi_min_internal_, dxi_, smooth_a_, dt_;
    int KL_, beam_ngp_, neutralize_, steps_;
    long lost_plasma_;
    std::vector<SpeciesRef*> species_;
    std::vector<BeamRef*> beams_;
    qz_sweep_params params_;
    View3D bsrc, fld, diag;
    void qz_setup();
    void snippet2(int KL);
    void snippet5(int rank, int n, MPI_Comm comm, int M);
    void snippet6();
    void snippet8(qz_sim* sim);
};

struct Beam {
    double *d_x_, *d_y_, *d_px_, *d_py_, *d_pz_, *d_xi_, *d_w_, *d_src_, *d_fld_;
    size_t n_; double q_, m_, xi_min_, dxi_;
    int KL_, ngp_, modes_, started_;
    qz_grid* qz_grid_;
    bool analytic_, parsed_, an_flat_;
    double an_n0_, an_sr_, an_xi0_, an_sxi_, an_len_, an_cut_head_, an_x0_, an_y0_, an_xs_, an_ys_, an_gamma_;
    qz_beam_view qz_view();
    void deposit(const View3D& src) const;
    void push(const View3D& fld, Real dt_kick, Real dt_drift, const View3D&, const View3D&, int);
    void snippet4(const qz_box& box);
};
"""

# where each snippet goes: file scope, or the body of a stub member / free function
WRAP = {
    1: None,
    2: "void Simulation::snippet2(int KL) {\n%s\n}",
    3: None,
    4: "void Beam::snippet4(const qz_box& box) {\n%s\n}",
    5: "void Simulation::snippet5(int rank, int n, MPI_Comm comm, int M) {\n%s\n}",
    6: "void Simulation::snippet6() {\n%s\n}",
    7: ("void snippet7(std::vector<Instance>& instances, size_t total_moments, int steps, double dt) {\n%s\n}"),
    8: "void Simulation::snippet8(qz_sim* sim) {\n%s\n}",
}


def _snippets():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```cpp\n(.*?)```", text, flags=re.S)


def test_snippets_are_all_wrapped():
    assert len(_snippets()) == len(WRAP)


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_snippets_compile(tmp_path):
    parts = [STUBS]
    for i, code in enumerate(_snippets(), start=1):
        if i == 8:          # a file-scope seed function, then the fragment that uses it
            head, sep, body = code.partition("#endif\n#ifdef QUARZ_B200\n")
            assert sep, "snippet 8: the seed function and the call are separate #ifdef blocks"
            parts.append(head + "#endif\n")
            parts.append(WRAP[8] % ("#ifdef QUARZ_B200\n" + body))
        elif WRAP[i] is None:
            parts.append(code)
        else:
            parts.append(WRAP[i] % code)
    src = tmp_path / "snippets.cpp"
    src.write_text("\n".join(parts))
    cuda = "/usr/local/cuda/include"
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-variable", "-Wno-unused-function",
           "-DQUARZ_B200", "-I", os.path.join(ROOT, "include"), "-I", cuda, str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
