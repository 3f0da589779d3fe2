// Device engine: owns the GPU state of one propagation problem (model, tables,
// wavefields, snapshots) and runs the time loops on a CUDA stream.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_ops.h"

namespace fwi {

struct FwiError : std::runtime_error {
    int code;
    FwiError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Device buffer (RAII).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    explicit DevBuf(size_t n);
    ~DevBuf();
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept;
    void alloc(size_t n);
    void zero(void *stream = nullptr);
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Static description of a propagation problem.
struct Problem {
    int nmodels;     // 2, 3, 6
    int nx, ny, nz;
    float dx, dy, dz;
    float dt;
    int nt;          // propagation samples (steps + 1)
    int sub;         // snapshot interval (0: none)
    int bc[6];
    int taper[6];
    float taper_strength;
    float free_surface_stiffness;
    bool grad_fp64 = true;
    int ncomp() const { return nmodels == 2 ? 1 : 3; }
    int64_t nxyz() const { return (int64_t)nx * ny * nz; }
};

// Injection / extraction tables on the device.
struct DevInj {
    int n[3] = {0, 0, 0};
    DevBuf gidx[3], trace[3], w[3];
    int ntrace = 0;
};
struct DevExt {
    int nrec = 0;
    DevBuf gidx, w;
};

class Engine {
public:
    Engine(int device, const Problem &pb);
    ~Engine();

    // Converted model [nmodels][nxyz] (host), boundary divisors and taper tables are built here.
    void set_model(const float *conv_model);

    // Forward propagation of one shot.  src: [ntrace][nt] (host, propagation
    // sampling); rcv out: [nrcomp][nrec][nt] (host).  When store is set and
    // sub > 0 the snapshots for a later adjoint are kept on the device.
    void forward(const InjTable &inj, int ntrace_src, const float *src, const ExtTable &ext, int nrcomp, float *rcv,
                 bool store);

    // Adjoint propagation + imaging; adj_src: [ntrace][nt]; grad out: [min(3,nm)][nxyz]
    // (host, float, before H quadrature and chain rule).
    void adjoint(const InjTable &inj, int ntrace_src, const float *adj_src, float *grad);

    bool has_snapshots() const { return snaps_valid_; }
    int64_t device_bytes() const;
    void sync();

private:
    void upload_inj(const InjTable &t, int ntrace, DevInj &d);
    void init_prev(const DevInj &inj, const float *src_dev, float *prev[3]);
    void step(int it, float *prev[3], float *curr[3], float *next[3], bool taper_prev);
    void inject(const DevInj &inj, const float *src_dev, int it, float *next[3]);
    void extract(const DevExt &ext, float *curr[3], float *rcv_dev, int nrcomp, int it);
    void image(int itl, float *curr[3], float *prevs[3]);

    int device_;
    Problem pb_;
    void *stream_ = nullptr;
    DevBuf model_;                 // [nm][nxyz]
    DevBuf fields_;                // 3 levels x ncomp x nxyz
    DevBuf aux_;                   // elastic derivative scratch
    DevBuf snaps_;                 // [nsnap][ncomp][nxyz]
    int nsnap_ = 0;
    bool snaps_valid_ = false;
    DevBuf grad_;                  // [3][nxyz] double
    DevBuf sdiv_;                  // boundary divisors, packed
    const float *sdiv_ptr_[6][3] = {};
    DevBuf taper_;                 // packed taper tables
    const float *taper_ptr_[6] = {};
    int scale_ = 0;
    DevBuf src_dev_, rcv_dev_;
    DevInj inj_;
    DevExt ext_;
};

}  // namespace fwi
