// bbmg_linsol.hpp -- C++ host-side mirror of NGA2's linear-solver object for
// the bbmg methods, over the C ABI of include/bbmg_b200.h.
//
// NGA2's flow solvers program against `linsol` (src/solver/linsol_class.f90:
// 16-58): they fill the public stencil map `stc`, the operator `opr`, `rhs` and
// `sol`, set `maxit`/`rcvg`, call init/setup/solve and read `it`/`rerr`.  This
// class keeps those names, that call order and the reference's error rules:
// setup before init and solve before setup are errors (ils_class.f90:684), an
// unknown method is an error (ils_class.f90:222), non-convergence is not.
// Arrays are owned by the object, laid out as the Fortran arrays
// (stencil index fastest, then i, j, k, with `no` overlap layers).
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/bbmg_b200.h"

namespace nga2 {

class bbmg_linsol {
  public:
    // ILS method ids (ils_class.f90:16-17)
    static constexpr int bbox = BBMG_METHOD_BBOX;
    static constexpr int pcg_bbox = BBMG_METHOD_PCG_BBOX;

    std::string name;
    int method = 0;
    int nst;
    std::vector<int> stc;      // nst x 3, stc[3*st + d]
    std::vector<double> opr;   // nst x (nx+2no) x (ny+2no) x (nz+2no)
    std::vector<double> rhs;   // (nx+2no) x (ny+2no) x (nz+2no)
    std::vector<double> sol;
    int maxit = 100;
    double rcvg = 1e-10;
    double acvg = 0.0;
    int it = -1;
    double rerr = 0.0, aerr = 0.0;
    bool setup_done = false;
    int precision = BBMG_PREC_FP64;

    bbmg_linsol(std::string nm, int nx, int ny, int nz, bool xper, bool yper, bool zper, int no, int nst_ = 7)
        : name(std::move(nm)), nst(nst_), stc(3 * nst_, 0) {
        grid_ = {nx, ny, nz, xper ? 1 : 0, yper ? 1 : 0, zper ? 1 : 0, no};
        size_t cells = (size_t)(nx + 2 * no) * (ny + 2 * no) * (nz + 2 * no);
        opr.assign(cells * nst, 0.0);
        rhs.assign(cells, 0.0);
        sol.assign(cells, 0.0);
    }
    ~bbmg_linsol() { destroy(); }
    bbmg_linsol(const bbmg_linsol &) = delete;
    bbmg_linsol &operator=(const bbmg_linsol &) = delete;

    // init: grid and stencil (ils_class.f90:162-226)
    void init(int method_) {
        if (method_ != bbox && method_ != pcg_bbox) throw std::invalid_argument("[bbmg_linsol init] Unknown solution method");
        destroy();
        method = method_;
        bbmg_params p;
        bbmg_default_params(&p);
        p.method = method;
        p.precision = precision;
        p.maxit = maxit;
        p.rcvg = rcvg;
        check(bbmg_create(&grid_, &p, &h_), nullptr);
    }
    // setup: every time the operator changes (ils_class.f90:230-376)
    void setup() {
        if (!h_) throw std::logic_error("[bbmg_linsol setup] init has not been called");
        check(bbmg_setup(h_, nst, stc.data(), opr.data()), h_);
        setup_done = true;
    }
    // solve: rhs and the initial guess in sol (ils_class.f90:674-822)
    void solve() {
        if (!setup_done) throw std::logic_error("[bbmg_linsol solve] Solver has not been setup.");
        check(bbmg_set_convergence(h_, maxit, rcvg), h_);
        int st = bbmg_solve(h_, rhs.data(), sol.data(), &it, &rerr);
        if (st != BBMG_OK && st != BBMG_MAXIT && st != BBMG_STAGNATION) check(st, h_);
    }
    void destroy() {
        if (h_) bbmg_destroy(h_);
        h_ = nullptr;
        setup_done = false;
    }
    bbmg_handle *handle() const { return h_; }

  private:
    bbmg_grid grid_{};
    bbmg_handle *h_ = nullptr;
    static void check(int st, const bbmg_handle *h) {
        if (st != BBMG_OK) throw std::runtime_error(std::string("bbmg: ") + bbmg_last_error(h));
    }
};

}  // namespace nga2
