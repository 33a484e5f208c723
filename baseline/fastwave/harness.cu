// Timing harness for the reference's GPU path: rave-sim fast-wave's CUDA
// kernels (fast-wave/fwcuda/kernels.cu, through the wrappers of
// fwcuda/wrappers.hpp) and its cuFFT plan class FFT<S> (fast-wave/src/fft.cpp),
// both compiled unmodified from the reference checkout by build.py, driven by
// this file over the schedule of fast-wave's run_simulation_inner
// (fast-wave/src/simulation.cpp:375-549).
//
// fast-wave's own driver (simulation.cpp, config_parsing.cpp, main.cpp) needs
// yaml-cpp, spdlog and NpyCpp, which this machine does not have, so this file
// restates its schedule: the plane-wave source, then per element the
// element's sub-steps (transmission wrapper + propagate: FFT forward,
// propagate_convolve_step, FFT inverse with its scale), the gap to the next
// element, square_and_downsample at the end of each phase step, and the phase
// steps restarted from a device snapshot taken before the first element with
// several x positions. The reference's per-element device synchronisation and
// the per-call device allocation of the sample grid are kept.
//
// The workload comes in the engine's own descriptors (include/rsw.h), so both
// paths run the same configuration. Measurement only: nothing in the product
// links this file.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fft.hpp"       // fast-wave FFT<S> (cuFFT)
#include "wrappers.hpp"  // fast-wave kernel wrappers
#include "rsw.h"         // workload descriptors

namespace {

// fast-wave's constants (fast-wave/include/simulation.hpp:18-22)
constexpr double kH = 6.62607004e-34, kC0 = 299792458.0, kEv = 1.602176634e-19;

struct Fail {
    char msg[256];
};

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        Fail f;
        std::snprintf(f.msg, sizeof f.msg, "%s: %s", what, cudaGetErrorString(e));
        throw f;
    }
}

template <typename S> __global__ void fill_plane_wave(DevComplex<S> *u, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u[i].x = S(1);
        u[i].y = S(0);
    }
}

std::complex<double> factor(std::complex<double> db, double t, double wl) {
    return std::exp(db * std::complex<double>(0.0, 2.0 * M_PI * t / wl));
}

template <typename S> struct Runner {
    const rsw_sim_desc &d;
    SimParams p{};
    FFT<S> fft;
    DevComplex<S> *u = nullptr, *U = nullptr, *snap = nullptr;
    S *det = nullptr;
    int n_pix = 0;
    int64_t steps = 0;

    Runner(const rsw_sim_desc &desc, int nps) : d(desc), fft(size_t(desc.n)) {
        p.N = int(d.n);
        p.dx = d.dx;
        p.z_detector = d.z_detector;
        p.detector_size = d.detector_size;
        p.detector_pixel_size_x = d.pixel_size_x;
        p.detector_pixel_size_y = d.pixel_size_y;
        n_pix = int(d.detector_size / d.pixel_size_x);
        const size_t bytes = size_t(d.n) * sizeof(DevComplex<S>);
        check(cudaMalloc(&u, bytes), "malloc u");
        check(cudaMalloc(&U, bytes), "malloc U");
        if (nps > 1) check(cudaMalloc(&snap, bytes), "malloc snapshot");
        check(cudaMalloc(&det, size_t(std::max(n_pix, 1)) * sizeof(S)), "malloc detector");
    }
    ~Runner() {
        cudaFree(u);
        cudaFree(U);
        cudaFree(snap);
        cudaFree(det);
    }

    void propagate(double dz, double cut) {
        fft.forward(u, U);
        propagate_convolve_step<S>(U, p, dz, cut);
        fft.inverse(U, u);
        ++steps;
    }

    // one element at phase step `ps` (fast-wave/src/simulation.cpp:131-203)
    void apply(const rsw_element &e, const std::vector<std::complex<double>> &db, double cut, size_t ps) {
        check(cudaDeviceSynchronize(), "sync before element");
        const double xp = e.x_positions[e.n_x_positions > 1 ? ps : 0];
        if (e.type == RSW_EL_GRATING || e.type == RSW_EL_DBA_GRATING) {
            const double dz = e.thickness / e.nr_steps;
            const Complex<S> fa(factor(db[0], dz, p.wl)), fb(factor(db[1], dz, p.wl));
            for (int i = 0; i < e.nr_steps; ++i) {
                if (e.type == RSW_EL_GRATING) {
                    const S dc = S(e.dc[0] + i * (e.dc[1] - e.dc[0]) / e.nr_steps);
                    apply_grating_factors<S>(u, p, fa, fb, e.pitch, dc, xp);
                } else {
                    const S dc0 = S(e.dc[0] + i * (e.dc[1] - e.dc[0]) / e.nr_steps);
                    const S dc1 = S(e.dc1[0] + i * (e.dc1[1] - e.dc1[0]) / e.nr_steps);
                    apply_dba_grating_factors<S>(u, p, fa, fb, e.pitch, e.pitch1, dc0, dc1, xp);
                }
                propagate(dz, cut);
            }
            if (e.substrate_thickness > 0) {
                scale<S>(u, Complex<S>(factor(db[2], e.substrate_thickness, p.wl)), p.N);
                propagate(e.substrate_thickness, cut);
            }
        } else {
            // the sample grid and its deltabeta table (vacuum first) go to the
            // device for each application, as in the reference
            const size_t cells = size_t(e.grid_z) * size_t(e.grid_x);
            std::vector<DevComplex<double>> dbs(1 + db.size());
            dbs[0] = DevComplex<double>{0.0, 0.0};
            for (size_t m = 0; m < db.size(); ++m) dbs[m + 1] = DevComplex<double>{db[m].real(), db[m].imag()};
            int8_t *d_grid = nullptr;
            DevComplex<double> *d_db = nullptr;
            check(cudaMalloc(&d_grid, cells), "malloc sample");
            check(cudaMalloc(&d_db, dbs.size() * sizeof(DevComplex<double>)), "malloc deltabetas");
            check(cudaMemcpyAsync(d_grid, e.grid, cells, cudaMemcpyHostToDevice), "copy sample");
            check(cudaMemcpyAsync(d_db, dbs.data(), dbs.size() * sizeof(DevComplex<double>), cudaMemcpyHostToDevice),
                  "copy deltabetas");
            for (int64_t z = 0; z < e.grid_z; ++z) {
                apply_sample_factors<S>(u, p, e.pixel_size_z, d_grid, e.pixel_size_x, size_t(e.grid_x), d_db, int(z),
                                        xp);
                propagate(e.pixel_size_z, cut);
            }
            check(cudaDeviceSynchronize(), "sync after sample");
            cudaFree(d_grid);
            cudaFree(d_db);
        }
        check(cudaGetLastError(), "element");
    }

    double total_thickness(const rsw_element &e) const {
        return e.type == RSW_EL_SAMPLE ? e.pixel_size_z * double(e.grid_z) : e.thickness + e.substrate_thickness;
    }
    double next_z(int i) const { return i + 1 < d.n_elements ? d.elements[i + 1].z_start : d.z_detector; }

    void detect(std::vector<S> &host, double *acc, double weight) {
        square_and_downsample<S>(u, p.N, det, n_pix, p.detector_pixel_size_x, p.detector_pixel_size_y, p.z_detector,
                                 p.dx);
        check(cudaMemcpy(host.data(), det, size_t(n_pix) * sizeof(S), cudaMemcpyDeviceToHost), "copy detector");
        for (int j = 0; j < n_pix; ++j) acc[j] += weight * double(host[j]);
    }

    // one source: fast-wave run_simulation_inner with a plane-wave source
    void run(const rsw_source_run &r, double src_z, int nps, double *acc) {
        p.wl = r.wavelength_m > 0 ? r.wavelength_m : kH * kC0 / (r.energy_ev * kEv);
        const double tol = 1e-8;
        // deltabeta per element in the engine's order (gratings a, b,
        // substrate; samples material 1..n)
        std::vector<std::vector<std::complex<double>>> db(size_t(std::max(d.n_elements, 1)));
        int64_t k = 0;
        for (int i = 0; i < d.n_elements; ++i) {
            const int cnt = d.elements[i].type == RSW_EL_SAMPLE ? d.elements[i].n_materials : 3;
            for (int m = 0; m < cnt; ++m, ++k) db[i].emplace_back(r.deltabeta[2 * k], r.deltabeta[2 * k + 1]);
        }
        auto cut = [&](int i) { return std::sin(d.cutoff_angles[i]) / p.wl; };
        std::vector<S> host(size_t(std::max(n_pix, 1)));
        const size_t bytes = size_t(d.n) * sizeof(DevComplex<S>);

        fill_plane_wave<S><<<1184, 256>>>(u, p.N);
        double z = d.n_elements > 0 ? d.elements[0].z_start : d.z_detector;
        if (z - src_z > 0) propagate(z - src_z, cut(0));
        int snap_el = -1;
        for (int i = 0; i < d.n_elements; ++i) {
            const rsw_element &e = d.elements[i];
            if (e.n_x_positions > 1 && snap_el < 0) {
                snap_el = i;
                check(cudaMemcpy(snap, u, bytes, cudaMemcpyDeviceToDevice), "snapshot");
            }
            apply(e, db[i], cut(i + 1), 0);
            z = e.z_start + total_thickness(e);
            const double rem = next_z(i) - z;
            if (rem > tol) {
                propagate(rem, cut(i + 1));
                z = next_z(i);
            }
        }
        detect(host, acc, r.weight);
        for (int ps = 1; ps < nps && snap_el >= 0; ++ps) {
            check(cudaDeviceSynchronize(), "sync before phase step");
            if (ps < nps - 1) check(cudaMemcpy(u, snap, bytes, cudaMemcpyDeviceToDevice), "restore");
            else std::swap(u, snap);
            for (int i = snap_el; i < d.n_elements; ++i) {
                const rsw_element &e = d.elements[i];
                apply(e, db[i], cut(i + 1), size_t(ps));
                z = e.z_start + total_thickness(e);
                const double rem = next_z(i) - z;
                if (rem > tol) {
                    propagate(rem, cut(i + 1));
                    z = next_z(i);
                }
            }
            detect(host, acc + size_t(ps) * size_t(n_pix), r.weight);
        }
        if (snap_el >= 0 && nps > 1) std::swap(u, snap);  // the last phase step swapped them
    }
};

template <typename S>
void run_all(const rsw_sim_desc &d, const rsw_source_run *runs, int n_runs, double src_z, int nps, int repeats,
             double *det, double *ms, int64_t *steps) {
    Runner<S> R(d, nps);
    const size_t np = size_t(std::max(R.n_pix, 1));
    std::vector<double> acc(size_t(nps) * np);
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "event");
    check(cudaEventCreate(&b), "event");
    for (int rep = 0; rep < repeats; ++rep) {
        std::fill(acc.begin(), acc.end(), 0.0);
        R.steps = 0;
        check(cudaDeviceSynchronize(), "sync");
        check(cudaEventRecord(a), "record");
        for (int i = 0; i < n_runs; ++i) R.run(runs[i], src_z, nps, acc.data());
        check(cudaEventRecord(b), "record");
        check(cudaEventSynchronize(b), "sync");
        float t = 0;
        check(cudaEventElapsedTime(&t, a, b), "elapsed");
        ms[rep] = t;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *steps = R.steps;
    std::copy(acc.begin(), acc.end(), det);
}

}  // namespace

extern "C" {

// Run `n_runs` plane-wave sources (source at z = src_z) of the workload `d`
// `repeats` times on the current device; det receives the weighted detector
// sum [phase][pix] of the last repeat (FP64 accumulation of fast-wave's
// per-source detector output), ms the device time of each repeat (CUDA
// events around the whole run, the reference's syncs included), steps the
// split steps of one repeat. nps: phase steps. Returns 0, or -1 with the
// message in err.
int fwh_run(const rsw_sim_desc *d, const rsw_source_run *runs, int n_runs, double src_z, int nps, int repeats,
            double *det, double *ms, int64_t *steps, char *err, int errlen) {
    try {
        if (d->n > (int64_t(1) << 30)) throw Fail{"fast-wave indexes fields with int: N > 2^30 is out of its range"};
        if (d->dtype == RSW_C128)
            run_all<double>(*d, runs, n_runs, src_z, nps, repeats, det, ms, steps);
        else
            run_all<float>(*d, runs, n_runs, src_z, nps, repeats, det, ms, steps);
        return 0;
    } catch (const Fail &f) {
        std::snprintf(err, size_t(errlen), "%s", f.msg);
        return -1;
    }
}

int fwh_detector_pixels(const rsw_sim_desc *d) { return int(d->detector_size / d->pixel_size_x); }

}  // extern "C"
