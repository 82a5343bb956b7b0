// tslb_run.cpp -- the host driver: the time loop of the reference's
// recursive_2c_TSLB3D.f90 (:344-844) over the C-ABI of libtslb.so.
//
//   tslb_run --workload droplet|jet [--n N] [--steps K] [--stamp S] [--stamp2d S2]
//            [--dump D] [--out DIR] [--load FILE] [--seed SEED] [--quiet]
//
// Per step, as the reference: one TSLB step (moments, collision with
// recursive reconstruction, streaming and boundary conditions, :346-838);
// every `stamp` steps the phi frame as VTK ImageData (print_vtk_phionly_sync,
// :582-590) and the FP64 diagnostics; every `stamp2d` steps the mid-plane
// slices of phi, u, v, w (print_raw_slice_2c_sync, :594-599); every `dump`
// steps a checkpoint (dump_distros_1c_3d, :600-605).  At the end it prints
// the reference's throughput line, glups = nx ny nz nsteps / 1e9 / wall
// seconds (:844), and the same over the stepping alone.
//
// Frames and slices are written asynchronously: the fields are downloaded
// into host buffers of their own and a writer thread writes the files while
// the lattice keeps stepping (at most two frames in flight).  Checkpoints are
// written synchronously.  The wall time includes waiting for the last write.
//
// Workloads: "droplet" is the static droplet of config 1 (colour mode,
// periodic n^3 box, R = n/4, tau 0.8, sigma 0.01, beta 0.7, phi =
// tanh((R - r)/2)); "jet" is the round jet of config 5 (192 x 192 x 384
// scaled by n/192, disc inlet refreshed every 10 steps on the device,
// pressure outlet behind a sponge layer).
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tslb.h"
#include "../../include/tslb_io.h"

namespace {

struct Options {
    std::string workload = "droplet", out = "output", load;
    int n = 64, steps = 2000, stamp = 500, stamp2d = 0, dump = 0;
    unsigned long long seed = 13;
    bool quiet = false;
};

int usage() {
    std::fprintf(stderr,
                 "usage: tslb_run --workload droplet|jet [--n N] [--steps K] [--stamp S] [--stamp2d S2]\n"
                 "                [--dump D] [--out DIR] [--load FILE] [--seed SEED] [--quiet]\n");
    return 2;
}

bool parse(int argc, char** argv, Options& o) {
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&](const char* what) -> const char* {
            if (i + 1 >= argc) { std::fprintf(stderr, "%s needs a value\n", what); return nullptr; }
            return argv[++i];
        };
        const char* v = nullptr;
        if (a == "--quiet") { o.quiet = true; continue; }
        if (!(v = next(a.c_str()))) return false;
        if (a == "--workload") o.workload = v;
        else if (a == "--n") o.n = std::atoi(v);
        else if (a == "--steps") o.steps = std::atoi(v);
        else if (a == "--stamp") o.stamp = std::atoi(v);
        else if (a == "--stamp2d") o.stamp2d = std::atoi(v);
        else if (a == "--dump") o.dump = std::atoi(v);
        else if (a == "--out") o.out = v;
        else if (a == "--load") o.load = v;
        else if (a == "--seed") o.seed = std::strtoull(v, nullptr, 10);
        else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); return false; }
    }
    return (o.workload == "droplet" || o.workload == "jet") && o.n >= 8 && o.steps >= 0;
}

int check(tslb_ctx* ctx, int rc, const char* what) {
    if (rc != TSLB_OK) std::fprintf(stderr, "tslb_run: %s failed (%d): %s\n", what, rc, tslb_last_error(ctx));
    return rc;
}

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// One thread that runs file-writing jobs in order; the first failing job's
// code is kept and returned by finish().
class Writer {
   public:
    Writer() : th_([this] { run(); }) {}
    ~Writer() { finish(); }
    void push(std::function<int()> job) {
        std::lock_guard<std::mutex> lk(mu_);
        q_.push_back(std::move(job));
        cv_.notify_one();
    }
    // block until fewer than n jobs are queued or running
    void wait_below(size_t n) {
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return q_.size() + busy_ < n; });
    }
    int finish() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_one();
        if (th_.joinable()) th_.join();
        return err_;
    }

   private:
    void run() {
        for (;;) {
            std::function<int()> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;
                job = std::move(q_.front());
                q_.pop_front();
                busy_ = 1;
            }
            const int rc = job();
            std::lock_guard<std::mutex> lk(mu_);
            if (rc && !err_) err_ = rc;
            busy_ = 0;
            done_.notify_all();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::deque<std::function<int()>> q_;
    size_t busy_ = 0;
    bool stop_ = false;
    int err_ = 0;
    std::thread th_;
};

}  // namespace

int main(int argc, char** argv) {
    Options o;
    if (!parse(argc, argv, o)) return usage();
    mkdir(o.out.c_str(), 0755);

    tslb_params p;
    tslb_default_params(&p);
    p.mode = TSLB_MODE_COLOUR;
    int nx, ny, nz;
    // jet geometry (scaled from 192 x 192 x 384, diameter 16)
    const double js = o.n / 192.0;
    float jet_d = 0.f, jet_w = 0.08f, jet_amp = 0.03f;
    if (o.workload == "droplet") {
        nx = ny = nz = o.n;
        p.tau_a = p.tau_b = 0.8f;
        p.sigma = 0.01f;
        p.beta = 0.7f;
        p.grad_threshold = 1e-3f;
    } else {
        nx = ny = o.n;
        nz = 2 * o.n;
        jet_d = (float)(16.0 * js);
        p.tau_a = p.tau_b = 3.0f * 8e-4f + 0.5f;
        p.sigma = 0.002f;
        p.beta = 0.7f;
        p.grad_threshold = 1e-3f;
        for (int f = 0; f < 4; ++f) p.bc[f] = TSLB_BC_PERIODIC;
        p.bc[4] = TSLB_BC_INLET;
        p.bc[5] = TSLB_BC_PRESSURE;
        for (int f = 0; f < 6; ++f) p.bc_phi[f] = -1.f;
        p.wall_phi_mode = 1;
    }
    const long long n = (long long)nx * ny * nz;
    tslb_ctx* ctx = nullptr;
    if (check(nullptr, tslb_create(&p, nx, ny, nz, &ctx), "tslb_create")) return 1;

    // initial state (recursive_2c_TSLB3D.f90:87-287) or a checkpoint
    std::vector<float> F[11];
    for (auto& v : F) v.assign((size_t)n, 0.f);
    enum { RHO = 0, U, V, W, PXX, PXY, PXZ, PYY, PYZ, PZZ, PHI };
    std::fill(F[RHO].begin(), F[RHO].end(), 1.f);
    if (o.workload == "droplet") {
        const double c = (o.n - 1) / 2.0, R = o.n / 4.0;
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const double r = std::sqrt((x - c) * (x - c) + (y - c) * (y - c) + (z - c) * (z - c));
                    F[PHI][x + (size_t)nx * (y + (size_t)ny * z)] = (float)std::tanh((R - r) / 2.0);
                }
    } else {
        std::fill(F[PHI].begin(), F[PHI].end(), -1.f);
        // sponge over the last 15% of the length: dtau = 0.3 s^2
        std::vector<float> sponge((size_t)n, 0.f);
        const double z0 = 0.85 * nz;
        for (int z = 0; z < nz; ++z) {
            const double zc = z + 0.5, s = zc > z0 ? (zc - z0) / (nz - z0) : 0.0;
            const float v = (float)(0.3 * s * s);
            for (size_t i = (size_t)z * nx * ny; i < (size_t)(z + 1) * nx * ny; ++i) sponge[i] = v;
        }
        if (check(ctx, tslb_set_tau_correction(ctx, sponge.data()), "tslb_set_tau_correction")) return 1;
    }
    if (!o.load.empty()) {
        if (check(ctx, tslb_checkpoint_load(ctx, o.load.c_str()), "tslb_checkpoint_load")) return 1;
    } else if (check(ctx, tslb_upload_moments(ctx, F[RHO].data(), F[U].data(), F[V].data(), F[W].data(),
                                              F[PXX].data(), F[PXY].data(), F[PXZ].data(), F[PYY].data(),
                                              F[PYZ].data(), F[PZZ].data(), F[PHI].data()),
                     "tslb_upload_moments")) {
        return 1;
    }
    std::printf("tslb_run: %s %d x %d x %d, tau %.4f, sigma %.4f, beta %.2f, %d steps from step %lld\n",
                o.workload.c_str(), nx, ny, nz, p.tau_a, p.sigma, p.beta, o.steps, tslb_steps_done(ctx));

    int iframe = 0, iframe2d = 0;
    double t_io = 0.0;
    Writer writer;
    // two sets of frame buffers, used in turn; the writer runs its jobs in
    // order, so a set is free once at most the previous stamp's jobs are left
    // page-locked (tslb_host_alloc), so the downloads run at the full PCIe rate
    struct FrameBuf {
        float* f[4] = {nullptr, nullptr, nullptr, nullptr};   // phi, u, v, w
        ~FrameBuf() {
            for (float* p : f) tslb_host_free(p);
        }
        bool ensure(int k, long long n) {
            if (!f[k]) f[k] = static_cast<float*>(tslb_host_alloc((long long)sizeof(float) * n));
            return f[k] != nullptr;
        }
    };
    std::shared_ptr<FrameBuf> bufs[2] = {std::make_shared<FrameBuf>(), std::make_shared<FrameBuf>()};
    int ibuf = 0;
    size_t last_jobs = 0;
    const long long step0 = tslb_steps_done(ctx);
    const double t1 = now();
    for (int s = 1; s <= o.steps; ++s) {
        const long long step = step0 + s;
        if (o.workload == "jet" && (step - 1) % 10 == 0) {
            if (check(ctx, tslb_set_inlet_disc(ctx, 4, nx / 2.f - 0.5f, ny / 2.f - 0.5f, jet_d / 2, jet_w, jet_amp, o.seed,
                                               (unsigned long long)((step - 1) / 10)),
                      "tslb_set_inlet_disc"))
                return 1;
        }
        if (check(ctx, tslb_step(ctx, 1), "tslb_step")) return 1;
        const bool frame = o.stamp > 0 && step % o.stamp == 0;
        const bool slice = o.stamp2d > 0 && step % o.stamp2d == 0;
        const bool dump = o.dump > 0 && step % o.dump == 0;
        if (!(frame || slice || dump)) continue;
        // the steps queued so far are stepping time, not output time
        if (check(ctx, tslb_synchronize(ctx), "tslb_synchronize")) return 1;
        const double ti = now();
        char path[4096];
        if (frame || slice) {
            // fields of this frame in a buffer set of their own, written by the writer thread
            writer.wait_below(last_jobs + 1);
            std::shared_ptr<FrameBuf> fb = bufs[ibuf];
            ibuf ^= 1;
            size_t jobs = 0;
            for (int k = 0; k < (slice ? 4 : 1); ++k)
                if (!fb->ensure(k, n)) {
                    std::fprintf(stderr, "tslb_run: page-locked frame buffer allocation failed\n");
                    return 1;
                }
            if (check(ctx, tslb_download_moments(ctx, nullptr, slice ? fb->f[1] : nullptr, slice ? fb->f[2] : nullptr,
                                                 slice ? fb->f[3] : nullptr, nullptr, nullptr, nullptr, nullptr,
                                                 nullptr, nullptr, fb->f[0]),
                      "tslb_download_moments"))
                return 1;
            if (frame) {
                ++iframe;
                double red[TSLB_NREDUCE];
                if (check(ctx, tslb_reduce(ctx, red), "tslb_reduce")) return 1;
                if (!o.quiet)
                    std::printf("step : %8lld  mass %.9e  mass_a %.9e  mom_z %.6e  umax %.6e\n", step,
                                red[TSLB_RED_MASS], red[TSLB_RED_MASS_A], red[TSLB_RED_MOM_Z], red[TSLB_RED_UMAX]);
                tslb_frame_path(path, sizeof(path), o.out.c_str(), "out", "phi", iframe, "vti");
                const std::string vti(path);
                ++jobs;
                writer.push([vti, fb, nx, ny, nz] {
                    const int rc = tslb_write_vti(vti.c_str(), "phi", nx, ny, nz, 1, fb->f[0]);
                    if (rc) std::fprintf(stderr, "tslb_run: writing %s failed (%d)\n", vti.c_str(), rc);
                    return rc;
                });
            }
            if (slice) {
                ++iframe2d;
                const std::string dir = o.out;
                const int k2 = iframe2d;
                ++jobs;
                writer.push([dir, k2, fb, nx, ny, nz] {
                    const char* names[4] = {"phi", "u", "v", "w"};
                    const float* data[4] = {fb->f[0], fb->f[1], fb->f[2], fb->f[3]};
                    for (int k = 0; k < 4; ++k) {
                        const int rc = tslb_write_slices(dir.c_str(), names[k], k2, nx, ny, nz, data[k]);
                        if (rc) {
                            std::fprintf(stderr, "tslb_run: writing the %s slices failed (%d)\n", names[k], rc);
                            return rc;
                        }
                    }
                    return 0;
                });
            }
            last_jobs = jobs;
        }
        if (dump) {
            tslb_frame_path(path, sizeof(path), o.out.c_str(), "dump", "state", (int)step, "ckpt");
            if (!o.quiet) std::printf("dump step at : %8lld\n", step);
            if (check(ctx, tslb_checkpoint_save(ctx, path), "tslb_checkpoint_save")) return 1;
        }
        t_io += now() - ti;
    }
    if (check(ctx, tslb_synchronize(ctx), "tslb_synchronize")) return 1;
    if (writer.finish()) return 1;
    const double t2 = now();
    const double wall = t2 - t1;
    std::printf("glups: %.6f\n", (double)n * o.steps / 1e9 / wall);
    std::printf("glups (stepping only): %.6f  wall %.3f s  output %.3f s  launches %lld\n",
                (double)n * o.steps / 1e9 / std::max(wall - t_io, 1e-9), wall, t_io, tslb_launch_count(ctx));
    tslb_destroy(ctx);
    return 0;
}
