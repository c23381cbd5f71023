// C-ABI of libjfli_b200: plain pointers, sizes and a caller-owned error buffer.
// Every entry point validates its arguments, enqueues its kernels on `stream`
// (a cudaStream_t; 0 = legacy default stream) and returns 0 on success or one of the
// JFLI_E* codes with a message in `err`. Nothing throws across this boundary and
// nothing synchronises the device except where documented.
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/jfli_b200.h"

#include "internal.h"

namespace jfli {
static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace jfli

using jfli::MeshDims;

namespace {

int fail(char* err, size_t errlen, int code, const char* fmt, ...) {
  if (err && errlen) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, errlen, fmt, ap);
    va_end(ap);
  }
  return code;
}

int cuda_status(cudaError_t e, char* err, size_t errlen, const char* what) {
  if (e == cudaSuccess) return JFLI_OK;
  return fail(err, errlen, JFLI_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Particle kernels address a particle's three components with 32-bit unsigned offsets
// (3 p) and cells with 32-bit signed offsets, so one mesh holds at most (2^32 - 1) / 3
// cells (about 1130^3); batches are separate meshes.
bool dims_ok(int nx, int ny, int nz, int batch) {
  return nx > 0 && ny > 0 && nz > 0 && batch > 0 && batch <= 65535 &&
         (long long)nx * ny * nz <= 1431655765LL;
}

#define CHECK_DIMS(nx, ny, nz, batch)                                                                       \
  if (!dims_ok(nx, ny, nz, batch))                                                                          \
  return fail(err, errlen, JFLI_EINVAL, "invalid mesh shape (%d, %d, %d) x batch %d", nx, ny, nz, batch)

#define CHECK_FFT(nx, ny, nz)                                                                               \
  if (!jfli::mesh_fft_supported(nx, ny, nz))                                                               \
  return fail(err, errlen, JFLI_EUNSUPPORTED,                                                               \
              "mesh (%d, %d, %d) unsupported: each axis must be 2^a 3^b <= 4096 and nz even with nz/2 "    \
              "also 2^a 3^b",                                                                               \
              nx, ny, nz)

#define CHECK_STENCIL(nx, ny, nz)                                                                           \
  if ((nx) < 4 || (ny) < 4 || (nz) < 4)                                                                     \
  return fail(err, errlen, JFLI_EUNSUPPORTED, "the finite-difference force needs every axis >= 4 cells, got (%d, %d, %d)", \
              nx, ny, nz)

#define CHECK_PTR(p)                                                                                        \
  if (!(p)) return fail(err, errlen, JFLI_EINVAL, "null pointer argument '%s'", #p)
#define CHECK_ALIGN16(p)                                                                                  \
  if (((uintptr_t)(p)) % 16 != 0)                                                                        \
  return fail(err, errlen, JFLI_EINVAL, "%s must be 16-byte aligned (AoS float4 force mesh)", #p)

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t spec_bytes(const MeshDims& d) { return align256((size_t)d.spec_elems() * d.batch * sizeof(float2)); }
size_t mesh_bytes(const MeshDims& d) { return align256((size_t)d.cells() * d.batch * sizeof(float)); }

}  // namespace

extern "C" {

const char* jfli_version(void) { return "jfli-b200 0.1.0 (sm_100a)"; }

long long jfli_launch_count(void) { return jfli::g_launches.load(); }

int jfli_device_check(char* err, size_t errlen) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, err, errlen, "cudaGetDevice");
  int major = 0, minor = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  if (major != 10 || minor != 0)
    return fail(err, errlen, JFLI_EUNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a only", dev,
                major, minor);
  return JFLI_OK;
}

int jfli_mesh_supported(int nx, int ny, int nz) { return jfli::mesh_fft_supported(nx, ny, nz) ? 1 : 0; }

long long jfli_spectrum_elems(int nx, int ny, int nz) { return (long long)nx * ny * (nz / 2 + 1); }

int jfli_rfft3d(void* stream, const float* mesh, void* spec, int nx, int ny, int nz, int batch, char* err,
                size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(mesh);
  CHECK_PTR(spec);
  const MeshDims d{nx, ny, nz, batch};
  return cuda_status(jfli::rfft3d_forward(mesh, (float2*)spec, d, 0.0f, (cudaStream_t)stream), err, errlen,
                     "jfli_rfft3d");
}

int jfli_irfft3d(void* stream, void* spec, float* mesh, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(mesh);
  CHECK_PTR(spec);
  const MeshDims d{nx, ny, nz, batch};
  const float scale = 1.0f / ((float)nx * (float)ny * (float)nz);
  return cuda_status(jfli::rfft3d_inverse((float2*)spec, mesh, d, scale, (cudaStream_t)stream), err, errlen,
                     "jfli_irfft3d");
}

int jfli_paint_cic(void* stream, const float* pos, int absolute, const float* weights, float weight, float* mesh,
                   int accumulate, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(pos);
  CHECK_PTR(mesh);
  const MeshDims d{nx, ny, nz, batch};
  cudaStream_t s = (cudaStream_t)stream;
  if (!accumulate) {
    cudaError_t e = cudaMemsetAsync(mesh, 0, (size_t)d.cells() * batch * sizeof(float), s);
    if (e != cudaSuccess) return cuda_status(e, err, errlen, "jfli_paint_cic memset");
  }
  return cuda_status(jfli::cic_paint(pos, absolute, weights, weight, mesh, d, s), err, errlen, "jfli_paint_cic");
}

int jfli_readout_cic(void* stream, const float* pos, int absolute, const float* mesh, float* out, int nx, int ny,
                     int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(pos);
  CHECK_PTR(mesh);
  CHECK_PTR(out);
  const MeshDims d{nx, ny, nz, batch};
  return cuda_status(jfli::cic_readout(pos, absolute, mesh, out, d, (cudaStream_t)stream), err, errlen,
                     "jfli_readout_cic");
}

size_t jfli_poisson_workspace_bytes(int nx, int ny, int nz, int batch) {
  return spec_bytes(MeshDims{nx, ny, nz, batch});
}

int jfli_poisson_potential(void* stream, const float* rho, float rho_mean, float* pot, void* workspace,
                           size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(rho);
  CHECK_PTR(pot);
  CHECK_PTR(workspace);
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < spec_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, spec_bytes(d));
  return cuda_status(jfli::poisson_potential(rho, (float2*)workspace, pot, d, rho_mean, 1.0f, (cudaStream_t)stream),
                     err, errlen, "jfli_poisson_potential");
}

// PGD adjoint workspace: spectrum, density, potential, divergence, rho_bar meshes, then the
// float4 PGD force mesh and the float4 cotangent paint.
size_t jfli_pgd_adjoint_workspace_bytes(int nx, int ny, int nz, int batch) {
  const MeshDims d{nx, ny, nz, batch};
  return spec_bytes(d) + 4 * mesh_bytes(d) + 2 * align256(sizeof(float) * 4 * (size_t)d.cells() * d.batch);
}

namespace {
// lam_x += scale J^T u, J = dF/dx for F the CIC readout of the FD force mesh of the
// particles' own density through the Poisson operator (pgd false) or the PGD filter.
int force_vjp(void* stream, const float* disp, const float* u, float scale, bool pgd, float kl, float ks,
              float* lam_x, void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
              size_t errlen, const char* name) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(disp);
  CHECK_PTR(u);
  CHECK_PTR(lam_x);
  CHECK_PTR(workspace);
  CHECK_ALIGN16(workspace);
  if (pgd && !(kl >= 0.0f && ks > 0.0f)) return fail(err, errlen, JFLI_EINVAL, "PGD scales need kl >= 0 and ks > 0");
  const MeshDims d{nx, ny, nz, batch};
  const size_t need = jfli_pgd_adjoint_workspace_bytes(nx, ny, nz, batch);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  cudaStream_t s = (cudaStream_t)stream;
  char* w = (char*)workspace;
  float2* spec = (float2*)w;
  float* rho = (float*)(w + spec_bytes(d));
  float* pot = (float*)(w + spec_bytes(d) + mesh_bytes(d));
  float* div = (float*)(w + spec_bytes(d) + 2 * mesh_bytes(d));
  float* rho_bar = (float*)(w + spec_bytes(d) + 3 * mesh_bytes(d));
  float* force = (float*)(w + spec_bytes(d) + 4 * mesh_bytes(d));
  float* ubar = force + 4 * (size_t)d.cells() * d.batch;
  float* x = const_cast<float*>(disp);  // painted only: the pass writes no particle array
  // the force mesh at x, as the forward builds it
  cudaError_t e = jfli::zero_floats(rho, d.cells() * batch, s);
  if (e == cudaSuccess) e = jfli::kick_drift_paint(x, x, nullptr, 0.f, 0.f, JFLI_STEP_PAINT, 1.0f, rho, d, s);
  if (e == cudaSuccess)
    e = pgd ? jfli::pgd_potential(rho, spec, pot, d, 1.0f, kl, ks, 1.0f, s)
            : jfli::poisson_potential(rho, spec, pot, d, 1.0f, 1.0f, s);
  if (e == cudaSuccess) e = jfli::force_mesh(pot, force, 1.0f, d, s);
  // rho_bar = P(div paint(u)); lam_x += scale grad R[rho_bar + u . F]
  if (e == cudaSuccess) e = cudaMemsetAsync(ubar, 0, sizeof(float) * 4 * (size_t)d.cells() * d.batch, s);
  if (e == cudaSuccess) e = jfli::paint_vec4(disp, u, ubar, d, s);
  if (e == cudaSuccess) e = jfli::divergence_fd(ubar, 1.0f, nullptr, 0.0f, 2, 0, div, d, s);
  if (e == cudaSuccess)
    e = pgd ? jfli::pgd_potential(div, spec, rho_bar, d, 0.0f, kl, ks, 1.0f, s)
            : jfli::poisson_potential(div, spec, rho_bar, d, 0.0f, 1.0f, s);
  if (e == cudaSuccess) e = jfli::adjoint_position(disp, u, rho_bar, force, scale, lam_x, d, s);
  return cuda_status(e, err, errlen, name);
}
}  // namespace

int jfli_pgd_adjoint(void* stream, const float* disp, const float* u, float alpha, float kl, float ks, float* lam_x,
                     void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                     size_t errlen) {
  return force_vjp(stream, disp, u, alpha, true, kl, ks, lam_x, workspace, workspace_bytes, nx, ny, nz, batch, err,
                   errlen, "jfli_pgd_adjoint");
}

int jfli_force_adjoint(void* stream, const float* disp, const float* u, float scale, float* lam_x, void* workspace,
                       size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  return force_vjp(stream, disp, u, scale, false, 0.f, 1.f, lam_x, workspace, workspace_bytes, nx, ny, nz, batch, err,
                   errlen, "jfli_force_adjoint");
}

int jfli_pgd_potential(void* stream, const float* rho, float rho_mean, float kl, float ks, float* pot, void* workspace,
                       size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(rho);
  CHECK_PTR(pot);
  CHECK_PTR(workspace);
  if (!(kl >= 0.0f && ks > 0.0f)) return fail(err, errlen, JFLI_EINVAL, "PGD scales need kl >= 0 and ks > 0");
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < spec_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, spec_bytes(d));
  return cuda_status(
      jfli::pgd_potential(rho, (float2*)workspace, pot, d, rho_mean, kl, ks, 1.0f, (cudaStream_t)stream), err, errlen,
      "jfli_pgd_potential");
}

size_t jfli_pm_forces_workspace_bytes(int nx, int ny, int nz, int batch) {
  const MeshDims d{nx, ny, nz, batch};
  return mesh_bytes(d) + spec_bytes(d);
}

int jfli_pm_forces(void* stream, const float* pos, int absolute, float scale, float* forces, void* workspace,
                   size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(pos);
  CHECK_PTR(forces);
  CHECK_PTR(workspace);
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < jfli_pm_forces_workspace_bytes(nx, ny, nz, batch))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes,
                jfli_pm_forces_workspace_bytes(nx, ny, nz, batch));
  cudaStream_t s = (cudaStream_t)stream;
  float* rho = (float*)workspace;  // the potential overwrites the density in place
  float2* spec = (float2*)((char*)workspace + mesh_bytes(d));
  cudaError_t e = cudaMemsetAsync(rho, 0, (size_t)d.cells() * batch * sizeof(float), s);
  if (e == cudaSuccess) e = jfli::cic_paint(pos, absolute, nullptr, 1.0f, rho, d, s);
  if (e == cudaSuccess) e = jfli::poisson_potential(rho, spec, rho, d, 1.0f, 1.0f, s);
  if (e == cudaSuccess) e = jfli::cic_readout_gradient(pos, absolute, rho, forces, scale, d, s);
  return cuda_status(e, err, errlen, "jfli_pm_forces");
}

int jfli_readout_gradient(void* stream, const float* pos, int absolute, const float* pot, float scale, float* forces,
                          int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_PTR(pos);
  CHECK_PTR(pot);
  CHECK_PTR(forces);
  const MeshDims d{nx, ny, nz, batch};
  return cuda_status(jfli::cic_readout_gradient(pos, absolute, pot, forces, scale, d, (cudaStream_t)stream), err,
                     errlen, "jfli_readout_gradient");
}

int jfli_force_mesh(void* stream, const float* pot, float scale, float* force, int nx, int ny, int nz, int batch,
                    char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_PTR(pot);
  CHECK_PTR(force);
  CHECK_ALIGN16(force);
  const MeshDims d{nx, ny, nz, batch};
  return cuda_status(jfli::force_mesh(pot, force, scale, d, (cudaStream_t)stream), err, errlen, "jfli_force_mesh");
}

int jfli_kick_drift_paint(void* stream, float* disp, float* vel, const float* force, float kick, float drift,
                          int flags, float weight, float* rho, int nx, int ny, int nz, int batch, char* err,
                          size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(vel);
  if ((flags & ~(JFLI_STEP_KICK | JFLI_STEP_DRIFT | JFLI_STEP_PAINT | JFLI_STEP_CORRECT | JFLI_STEP_CLEAR)) != 0)
    return fail(err, errlen, JFLI_EINVAL, "unknown step flags 0x%x", flags);
  if ((flags & JFLI_STEP_KICK) && (flags & JFLI_STEP_CORRECT))
    return fail(err, errlen, JFLI_EINVAL, "KICK and CORRECT are exclusive");
  if ((flags & (JFLI_STEP_KICK | JFLI_STEP_CORRECT)) && !force)
    return fail(err, errlen, JFLI_EINVAL, "kick requested without a force mesh");
  if (force) CHECK_ALIGN16(force);
  if ((flags & JFLI_STEP_PAINT) && !rho) return fail(err, errlen, JFLI_EINVAL, "paint requested without a mesh");
  if ((flags & JFLI_STEP_CLEAR) && !(flags & JFLI_STEP_PAINT))
    return fail(err, errlen, JFLI_EINVAL, "CLEAR needs PAINT");
  const MeshDims d{nx, ny, nz, batch};
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaSuccess;
  // cleared right before the pass, so the zeroed lines are still in L2 when the deposits arrive
  if (flags & JFLI_STEP_CLEAR) e = jfli::zero_floats(rho, d.cells() * batch, s);
  if (e == cudaSuccess)
    e = jfli::kick_drift_paint(disp, vel, force, kick, drift, flags & ~JFLI_STEP_CLEAR, weight, rho, d, s);
  return cuda_status(e, err, errlen, "jfli_kick_drift_paint");
}

size_t jfli_pm_step_workspace_bytes(int nx, int ny, int nz, int batch) {
  const MeshDims d{nx, ny, nz, batch};
  return spec_bytes(d) + mesh_bytes(d);
}

int jfli_pm_step(void* stream, float* disp, float* vel, float kick, float drift, int flags, float* rho, float* force,
                 void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                 size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(disp);
  CHECK_PTR(vel);
  CHECK_PTR(rho);
  CHECK_PTR(force);
  CHECK_ALIGN16(force);
  CHECK_PTR(workspace);
  const MeshDims d{nx, ny, nz, batch};
  const size_t need = jfli_pm_step_workspace_bytes(nx, ny, nz, batch);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  if ((flags & ~(JFLI_STEP_KICK | JFLI_STEP_DRIFT | JFLI_STEP_FORCE)) != 0)
    return fail(err, errlen, JFLI_EINVAL, "unknown step flags 0x%x", flags);
  cudaStream_t s = (cudaStream_t)stream;
  float2* spec = (float2*)workspace;
  float* pot = (float*)((char*)workspace + spec_bytes(d));
  cudaError_t e = jfli::zero_floats(rho, d.cells() * batch, s);
  if (e == cudaSuccess)
    e = jfli::kick_drift_paint(disp, vel, force, kick, drift,
                               (flags & (JFLI_STEP_KICK | JFLI_STEP_DRIFT)) | JFLI_STEP_PAINT, 1.0f, rho, d, s);
  if (e == cudaSuccess && (flags & JFLI_STEP_FORCE)) e = jfli::poisson_potential(rho, spec, pot, d, 1.0f, 1.0f, s);
  if (e == cudaSuccess && (flags & JFLI_STEP_FORCE)) e = jfli::force_mesh(pot, force, 1.0f, d, s);
  return cuda_status(e, err, errlen, "jfli_pm_step");
}

int jfli_pm_step_slots(void* stream, float* disp, float* vel, const float* kicks, const float* drifts,
                       const int* slot_flags, float* rho, float* force, void* workspace, size_t workspace_bytes, int nx,
                       int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(disp);
  CHECK_PTR(vel);
  CHECK_PTR(kicks);
  CHECK_PTR(drifts);
  CHECK_PTR(slot_flags);
  CHECK_PTR(rho);
  CHECK_PTR(force);
  CHECK_ALIGN16(force);
  CHECK_PTR(workspace);
  const MeshDims d{nx, ny, nz, batch};
  const size_t need = jfli_pm_step_workspace_bytes(nx, ny, nz, batch);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  cudaStream_t s = (cudaStream_t)stream;
  float2* spec = (float2*)workspace;
  float* pot = (float*)((char*)workspace + spec_bytes(d));
  cudaError_t e = jfli::zero_floats(rho, d.cells() * batch, s);
  if (e == cudaSuccess) e = jfli::kick_drift_paint_slots(disp, vel, force, kicks, drifts, slot_flags, 1.0f, rho, d, s);
  if (e == cudaSuccess) e = jfli::poisson_potential(rho, spec, pot, d, 1.0f, 1.0f, s);
  if (e == cudaSuccess) e = jfli::force_mesh(pot, force, 1.0f, d, s);
  return cuda_status(e, err, errlen, "jfli_pm_step_slots");
}

int jfli_poisson_force(void* stream, float* rho, float rho_mean, int clear_rho, float scale, float* pot, float* force,
                       void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                       size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(rho);
  CHECK_PTR(pot);
  CHECK_PTR(force);
  CHECK_ALIGN16(force);
  CHECK_PTR(workspace);
  const MeshDims d{nx, ny, nz, batch};
  const size_t need = jfli_poisson_workspace_bytes(nx, ny, nz, batch);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  if (pot == rho && clear_rho) return fail(err, errlen, JFLI_EINVAL, "pot must not alias rho when clear_rho is set");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = jfli::poisson_potential(rho, (float2*)workspace, pot, d, rho_mean, 1.0f, s, clear_rho ? rho : nullptr);
  if (e == cudaSuccess) e = jfli::force_mesh(pot, force, scale, d, s);
  return cuda_status(e, err, errlen, "jfli_poisson_force");
}

int jfli_ic_filter(void* stream, const float* noise, float* out, const float* ktab, const float* ptab, int ntab,
                   float lx, float ly, float lz, int zero_mode_one, void* workspace, size_t workspace_bytes, int nx,
                   int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(noise);
  CHECK_PTR(out);
  CHECK_PTR(ktab);
  CHECK_PTR(ptab);
  CHECK_PTR(workspace);
  if (ntab < 2 || ntab > 4096) return fail(err, errlen, JFLI_EINVAL, "table length %d outside [2, 4096]", ntab);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < spec_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, spec_bytes(d));
  const float box[3] = {lx, ly, lz};
  return cuda_status(jfli::ic_filter(noise, (float2*)workspace, out, d, ktab, ptab, ntab, box, zero_mode_one,
                                     (cudaStream_t)stream),
                     err, errlen, "jfli_ic_filter");
}

size_t jfli_lpt_workspace_bytes(int nx, int ny, int nz, int batch) {
  const MeshDims d{nx, ny, nz, batch};
  return spec_bytes(d) + 2 * mesh_bytes(d) + align256((size_t)d.cells() * batch * 3 * sizeof(float));
}

int jfli_lpt(void* stream, const float* ic, int order, float c1x, float c2x, float c1p, float c2p, float* dx, float* p,
             void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(ic);
  CHECK_PTR(dx);
  CHECK_PTR(p);
  CHECK_PTR(workspace);
  if (order != 1 && order != 2) return fail(err, errlen, JFLI_EINVAL, "LPT order must be 1 or 2, got %d", order);
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < jfli_lpt_workspace_bytes(nx, ny, nz, batch))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes,
                jfli_lpt_workspace_bytes(nx, ny, nz, batch));
  cudaStream_t s = (cudaStream_t)stream;
  char* w = (char*)workspace;
  float2* spec = (float2*)w;
  float* pot = (float*)(w + spec_bytes(d));
  float* src = (float*)(w + spec_bytes(d) + mesh_bytes(d));
  float* f2 = (float*)(w + spec_bytes(d) + 2 * mesh_bytes(d));
  // first order: phi1 = laplace^-1 ic, F1 = -D phi1 at the grid points (written to dx)
  cudaError_t e = jfli::poisson_potential(ic, spec, pot, d, 0.0f, 1.0f, s);
  if (e == cudaSuccess) e = jfli::grid_gradient(pot, dx, 1.0f, 0, d, s);
  if (e == cudaSuccess && order == 2) {
    e = jfli::lpt2_source(dx, src, d, s);
    if (e == cudaSuccess) e = jfli::poisson_potential(src, spec, pot, d, 0.0f, 1.0f, s);
    if (e == cudaSuccess) e = jfli::grid_gradient(pot, f2, 1.0f, 0, d, s);
  }
  if (e == cudaSuccess) e = jfli::lpt_combine(dx, order == 2 ? f2 : nullptr, c1x, c2x, c1p, c2p, dx, p, d, s);
  return cuda_status(e, err, errlen, "jfli_lpt");
}

int jfli_lpt_lightcone(void* stream, const float* ic, int order, const double* tables, int n_chi, int n_g,
                       const double* background, float lx, float ly, float lz, float ox, float oy, float oz, float* dx,
                       float* p, float* a_out, void* workspace, size_t workspace_bytes, int nx, int ny, int nz,
                       int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(ic);
  CHECK_PTR(tables);
  CHECK_PTR(background);
  CHECK_PTR(dx);
  CHECK_PTR(p);
  CHECK_PTR(workspace);
  if (order != 1 && order != 2) return fail(err, errlen, JFLI_EINVAL, "LPT order must be 1 or 2, got %d", order);
  if (n_chi < 2 || n_g < 2) return fail(err, errlen, JFLI_EINVAL, "tables need at least 2 points");
  const MeshDims d{nx, ny, nz, batch};
  // F1 (and F2) need a mesh of three components each beyond the LPT workspace
  const size_t need = jfli_lpt_workspace_bytes(nx, ny, nz, batch) + align256(sizeof(float) * 3 * (size_t)d.cells() * batch);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  cudaStream_t s = (cudaStream_t)stream;
  char* w = (char*)workspace;
  float2* spec = (float2*)w;
  float* pot = (float*)(w + spec_bytes(d));
  float* src = (float*)(w + spec_bytes(d) + mesh_bytes(d));
  float* f2 = (float*)(w + spec_bytes(d) + 2 * mesh_bytes(d));
  float* f1 = (float*)(w + jfli_lpt_workspace_bytes(nx, ny, nz, batch));
  cudaError_t e = jfli::poisson_potential(ic, spec, pot, d, 0.0f, 1.0f, s);
  if (e == cudaSuccess) e = jfli::grid_gradient(pot, f1, 1.0f, 0, d, s);
  if (e == cudaSuccess && order == 2) {
    e = jfli::lpt2_source(f1, src, d, s);
    if (e == cudaSuccess) e = jfli::poisson_potential(src, spec, pot, d, 0.0f, 1.0f, s);
    if (e == cudaSuccess) e = jfli::grid_gradient(pot, f2, 1.0f, 0, d, s);
  }
  jfli::LptLightcone lc;
  lc.tables = tables;
  lc.n_chi = n_chi;
  lc.n_g = n_g;
  lc.box[0] = lx;
  lc.box[1] = ly;
  lc.box[2] = lz;
  lc.obs[0] = ox;
  lc.obs[1] = oy;
  lc.obs[2] = oz;
  lc.om = background[0];
  lc.ok = background[1];
  lc.ode = background[2];
  lc.w0 = background[3];
  lc.wa = background[4];
  if (e == cudaSuccess) e = jfli::lpt_combine_lightcone(f1, order == 2 ? f2 : nullptr, dx, p, a_out, lc, d, s);
  return cuda_status(e, err, errlen, "jfli_lpt_lightcone");
}

size_t jfli_lpt_lightcone_workspace_bytes(int nx, int ny, int nz, int batch) {
  const MeshDims d{nx, ny, nz, batch};
  return jfli_lpt_workspace_bytes(nx, ny, nz, batch) + align256(sizeof(float) * 3 * (size_t)d.cells() * batch);
}

size_t jfli_power_spectrum_workspace_bytes(int nx, int ny, int nz, int batch, int nedges) {
  const MeshDims d{nx, ny, nz, batch};
  const size_t partial = (size_t)jfli::x_pass_ctas(d) * batch * 3 * (nedges + 1) * sizeof(double);
  return spec_bytes(d) + align256(partial);
}

int jfli_power_spectrum(void* stream, const float* mesh, const float* kedges, int nedges, float lx, float ly,
                        float lz, double* out, void* workspace, size_t workspace_bytes, int nx, int ny, int nz,
                        int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(mesh);
  CHECK_PTR(kedges);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  if (nedges < 1 || nedges > 2048) return fail(err, errlen, JFLI_EINVAL, "nedges %d outside [1, 2048]", nedges);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  const size_t need = jfli_power_spectrum_workspace_bytes(nx, ny, nz, batch, nedges);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  cudaStream_t s = (cudaStream_t)stream;
  float2* spec = (float2*)workspace;
  double* partials = (double*)((char*)workspace + spec_bytes(d));
  const float box[3] = {lx, ly, lz};
  const float norm = 1.0f / ((float)nx * (float)ny * (float)nz);
  cudaError_t e = jfli::power_partials(mesh, spec, partials, d, kedges, nedges, box, norm, s);
  if (e == cudaSuccess) e = jfli::power_finalize(partials, jfli::x_pass_ctas(d), nedges + 1, out, batch, s);
  return cuda_status(e, err, errlen, "jfli_power_spectrum");
}

size_t jfli_power_poles_workspace_bytes(int nx, int ny, int nz, int batch, int nedges, int nell, int cross) {
  if (nedges < 1 || nell < 1) return 0;
  const MeshDims d{nx, ny, nz, batch};
  return spec_bytes(d) * (cross ? 2 : 1) +
         align256(sizeof(double) * (size_t)(2 * nell + 2) * (nedges + 1) * jfli::power_poles_ctas(d) * batch);
}

int jfli_power_poles(void* stream, const float* mesh, const float* mesh2, const float* kedges, int nedges, float lx,
                     float ly, float lz, float losx, float losy, float losz, const int* ells, int nell, double* out,
                     void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                     size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(mesh);
  CHECK_PTR(kedges);
  CHECK_PTR(ells);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  if (nedges < 1 || nedges > 512) return fail(err, errlen, JFLI_EINVAL, "nedges %d outside [1, 512]", nedges);
  if (nell < 1 || nell > 8) return fail(err, errlen, JFLI_EINVAL, "%d multipoles outside [1, 8]", nell);
  for (int i = 0; i < nell; ++i)
    if (ells[i] < 0 || ells[i] > 16) return fail(err, errlen, JFLI_EINVAL, "multipole %d outside [0, 16]", ells[i]);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  const size_t need = jfli_power_poles_workspace_bytes(nx, ny, nz, batch, nedges, nell, mesh2 != nullptr);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  float2* s1 = (float2*)workspace;
  float2* s2 = mesh2 ? (float2*)((char*)workspace + spec_bytes(d)) : nullptr;
  double* partials = (double*)((char*)workspace + spec_bytes(d) * (mesh2 ? 2 : 1));
  const float box[3] = {lx, ly, lz}, los[3] = {losx, losy, losz};
  return cuda_status(jfli::power_poles(mesh, mesh2, d, kedges, nedges, box, los, ells, nell, s1, s2, partials, out,
                                       (cudaStream_t)stream),
                     err, errlen, "jfli_power_poles");
}

int jfli_healpix_paint(void* stream, const float* disp, int absolute, const float* weights, float weight, float lx,
                       float ly, float lz, float ox, float oy, float oz, float rmin, float rmax, int nside, int scheme,
                       float* map, int accumulate, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(map);
  if (nside < 1 || nside > 8192) return fail(err, errlen, JFLI_EINVAL, "nside %d outside [1, 8192]", nside);
  if (scheme != JFLI_HEALPIX_NGP && scheme != JFLI_HEALPIX_BILINEAR)
    return fail(err, errlen, JFLI_EUNSUPPORTED, "HEALPix scheme %d not supported (0 = ngp, 1 = bilinear)", scheme);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  cudaStream_t s = (cudaStream_t)stream;
  if (!accumulate) {
    cudaError_t e = cudaMemsetAsync(map, 0, (size_t)12 * nside * nside * batch * sizeof(float), s);
    if (e != cudaSuccess) return cuda_status(e, err, errlen, "jfli_healpix_paint memset");
  }
  const float box[3] = {lx, ly, lz};
  const float obs[3] = {ox, oy, oz};
  return cuda_status(
      jfli::healpix_paint(disp, absolute, weights, weight, d, box, obs, rmin, rmax, nside, scheme, map, s), err,
      errlen, "jfli_healpix_paint");
}

int jfli_healpix_paint_shells(void* stream, const float* disp, int absolute, const float* weights, float weight,
                              float lx, float ly, float lz, float ox, float oy, float oz, int nshells,
                              const double* rmin, const double* rmax, const float* scale, int nside, int scheme,
                              float sigma, float* maps, int accumulate, int nx, int ny, int nz, int batch, char* err,
                              size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(maps);
  if (batch != 1) return fail(err, errlen, JFLI_EUNSUPPORTED, "one particle set per call (batch %d)", batch);
  if (nshells < 1) return fail(err, errlen, JFLI_EINVAL, "nshells must be >= 1");
  CHECK_PTR(rmin);
  CHECK_PTR(rmax);
  CHECK_PTR(scale);
  if (nside < 1 || nside > 8192) return fail(err, errlen, JFLI_EINVAL, "nside %d outside [1, 8192]", nside);
  if (scheme != JFLI_HEALPIX_NGP && scheme != JFLI_HEALPIX_BILINEAR && scheme != 2)
    return fail(err, errlen, JFLI_EUNSUPPORTED, "HEALPix scheme %d not supported (0 ngp, 1 bilinear, 2 rbf_neighbor)",
                scheme);
  if (scheme == 2 && !(sigma > 0.f && sigma < 3.2f))
    return fail(err, errlen, JFLI_EINVAL, "rbf_neighbor sigma %g outside (0, pi)", (double)sigma);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  cudaStream_t s = (cudaStream_t)stream;
  if (!accumulate) {
    cudaError_t e = cudaMemsetAsync(maps, 0, (size_t)12 * nside * nside * nshells * sizeof(float), s);
    if (e != cudaSuccess) return cuda_status(e, err, errlen, "jfli_healpix_paint_shells memset");
  }
  const float box[3] = {lx, ly, lz};
  const float obs[3] = {ox, oy, oz};
  return cuda_status(jfli::healpix_paint_shells(disp, absolute, weights, weight, d, box, obs, nshells, rmin, rmax,
                                                scale, nside, scheme, maps, s, scheme == 2 ? sigma : 0.f),
                     err, errlen, "jfli_healpix_paint_shells");
}

int jfli_healpix_paint_shells_adjoint(void* stream, const float* disp, int absolute, const float* weights,
                                      float weight, float lx, float ly, float lz, float ox, float oy, float oz,
                                      int nshells, const double* rmin, const double* rmax, const float* scale,
                                      int nside, int scheme, const float* maps_bar, float* disp_bar,
                                      float* weights_bar, int nx, int ny, int nz, int batch, char* err,
                                      size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(maps_bar);
  CHECK_PTR(disp_bar);
  if (batch != 1) return fail(err, errlen, JFLI_EUNSUPPORTED, "one particle set per call (batch %d)", batch);
  if (nshells < 1) return fail(err, errlen, JFLI_EINVAL, "nshells must be >= 1");
  CHECK_PTR(rmin);
  CHECK_PTR(rmax);
  CHECK_PTR(scale);
  if (nside < 1 || nside > 8192) return fail(err, errlen, JFLI_EINVAL, "nside %d outside [1, 8192]", nside);
  if (scheme != JFLI_HEALPIX_NGP && scheme != JFLI_HEALPIX_BILINEAR)
    return fail(err, errlen, JFLI_EUNSUPPORTED, "the shell-painting adjoint has the ngp (0) and bilinear (1) schemes, "
                "not %d", scheme);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  const float box[3] = {lx, ly, lz};
  const float obs[3] = {ox, oy, oz};
  return cuda_status(jfli::healpix_paint_shells_adjoint(disp, absolute, weights, weight, d, box, obs, nshells, rmin,
                                                        rmax, scale, nside, scheme, maps_bar, disp_bar, weights_bar,
                                                        (cudaStream_t)stream),
                     err, errlen, "jfli_healpix_paint_shells_adjoint");
}

int jfli_healpix_paint_rbf(void* stream, const float* disp, int absolute, const float* weights, float weight,
                           float lx, float ly, float lz, float ox, float oy, float oz, float rmin, float rmax, int nside,
                           float sigma, float* map, int accumulate, int nx, int ny, int nz, int batch, char* err,
                           size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(map);
  if (nside < 1 || nside > 8192) return fail(err, errlen, JFLI_EINVAL, "nside %d outside [1, 8192]", nside);
  if (!(sigma > 0.f) || !(sigma < 3.2f)) return fail(err, errlen, JFLI_EINVAL, "kernel sigma must be in (0, pi) radians");
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  cudaStream_t s = (cudaStream_t)stream;
  if (!accumulate) {
    cudaError_t e = cudaMemsetAsync(map, 0, (size_t)12 * nside * nside * batch * sizeof(float), s);
    if (e != cudaSuccess) return cuda_status(e, err, errlen, "jfli_healpix_paint_rbf memset");
  }
  const float box[3] = {lx, ly, lz};
  const float obs[3] = {ox, oy, oz};
  return cuda_status(
      jfli::healpix_paint(disp, absolute, weights, weight, d, box, obs, rmin, rmax, nside, 2, map, s, sigma), err,
      errlen, "jfli_healpix_paint_rbf");
}

// Arguments of the replica painter and its adjoint (0 when valid).
static int tiled_args_check(const float* vel, float lx, float ly, float lz, int ntiles, const signed char* rotations,
                            const float* shifts, float t, float dbound, const float* chi, const float* a_chi,
                            int n_chi, const float* ga, const float* g, int n_g, const float* da, const float* dgfa,
                            int n_d, int nside, int scheme, char* err, size_t errlen) {
  CHECK_PTR(rotations);
  CHECK_PTR(shifts);
  if (nside < 1 || nside > 8192) return fail(err, errlen, JFLI_EINVAL, "nside %d outside [1, 8192]", nside);
  if (scheme != JFLI_HEALPIX_NGP && scheme != JFLI_HEALPIX_BILINEAR)
    return fail(err, errlen, JFLI_EUNSUPPORTED, "HEALPix scheme %d not supported (0 = ngp, 1 = bilinear)", scheme);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  if (ntiles < 1 || ntiles > jfli::kMaxTiles)
    return fail(err, errlen, JFLI_EINVAL, "ntiles %d outside [1, %d]", ntiles, jfli::kMaxTiles);
  for (int i = 0; i < ntiles; ++i) {  // signed permutation matrices only
    int used = 0;
    for (int r = 0; r < 3; ++r) {
      int nz_in_row = 0;
      for (int c = 0; c < 3; ++c) {
        const int m = rotations[9 * i + 3 * r + c];
        if (m == 0) continue;
        if ((m != 1 && m != -1) || (used & (1 << c)))
          return fail(err, errlen, JFLI_EINVAL, "tile %d: rotation is not a signed permutation matrix", i);
        used |= 1 << c;
        ++nz_in_row;
      }
      if (nz_in_row != 1) return fail(err, errlen, JFLI_EINVAL, "tile %d: rotation is not a signed permutation matrix", i);
    }
    for (int c = 0; c < 3; ++c)
      if (!isfinite(shifts[3 * i + c])) return fail(err, errlen, JFLI_EINVAL, "tile %d: shift is not finite", i);
  }
  if (vel) {
    CHECK_PTR(chi);
    CHECK_PTR(a_chi);
    CHECK_PTR(ga);
    CHECK_PTR(g);
    CHECK_PTR(da);
    CHECK_PTR(dgfa);
    if (n_chi < 2 || n_g < 2 || n_d < 2) return fail(err, errlen, JFLI_EINVAL, "tables need at least 2 entries");
    if (!(t > 0)) return fail(err, errlen, JFLI_EINVAL, "scale factor must be positive");
    if (!(dbound >= 0) || !isfinite(dbound)) return fail(err, errlen, JFLI_EINVAL, "drift bound must be finite, >= 0");
  }
  if (nside < 1 || nside > 8192) return fail(err, errlen, JFLI_EINVAL, "nside %d outside [1, 8192]", nside);
  if (scheme != JFLI_HEALPIX_NGP && scheme != JFLI_HEALPIX_BILINEAR)
    return fail(err, errlen, JFLI_EUNSUPPORTED, "HEALPix scheme %d not supported (0 = ngp, 1 = bilinear)", scheme);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  return 0;
}

int jfli_healpix_paint_tiled(void* stream, const float* disp, int absolute, const float* vel, const float* weights,
                             float weight, float lx, float ly, float lz, float ox, float oy, float oz, int ntiles,
                             const signed char* rotations, const float* shifts, int telephoto, float rmin, float rmax,
                             float t, float gp_t, float dbound, const float* chi, const float* a_chi, int n_chi,
                             const float* ga, const float* g, int n_g, const float* da, const float* dgfa, int n_d,
                             int nside, int scheme, float* map, int accumulate, int nx, int ny, int nz, int batch,
                             char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(map);
  if (int rc = tiled_args_check(vel, lx, ly, lz, ntiles, rotations, shifts, t, dbound, chi, a_chi, n_chi, ga, g,
                                n_g, da, dgfa, n_d, nside, scheme, err, errlen))
    return rc;
  const MeshDims d{nx, ny, nz, batch};
  cudaStream_t s = (cudaStream_t)stream;
  if (!accumulate) {
    cudaError_t e = cudaMemsetAsync(map, 0, (size_t)12 * nside * nside * batch * sizeof(float), s);
    if (e != cudaSuccess) return cuda_status(e, err, errlen, "jfli_healpix_paint_tiled memset");
  }
  const float box[3] = {lx, ly, lz};
  const float obs[3] = {ox, oy, oz};
  const jfli::DriftTables tb{chi, a_chi, n_chi, ga, g, n_g, da, dgfa, n_d};
  return cuda_status(jfli::healpix_paint_tiled(disp, absolute, vel, weights, weight, d, box, obs, ntiles, rotations,
                                               shifts, telephoto, rmin, rmax, t, gp_t, dbound, tb, nside, scheme, map,
                                               s),
                     err, errlen, "jfli_healpix_paint_tiled");
}

int jfli_healpix_paint_tiled_adjoint(void* stream, const float* disp, int absolute, const float* vel,
                                     const float* weights, float weight, float lx, float ly, float lz, float ox,
                                     float oy, float oz, int ntiles, const signed char* rotations, const float* shifts,
                                     int telephoto, float rmin, float rmax, float t, float gp_t, float dbound,
                                     const float* chi, const float* a_chi, int n_chi, const float* ga, const float* g,
                                     int n_g, const float* da, const float* dgfa, int n_d, int nside, int scheme,
                                     const float* map_bar, float* disp_bar, float* vel_bar, float* weights_bar,
                                     int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(map_bar);
  CHECK_PTR(disp_bar);
  if (int rc = tiled_args_check(vel, lx, ly, lz, ntiles, rotations, shifts, t, dbound, chi, a_chi, n_chi, ga, g,
                                n_g, da, dgfa, n_d, nside, scheme, err, errlen))
    return rc;
  const MeshDims d{nx, ny, nz, batch};
  const float box[3] = {lx, ly, lz};
  const float obs[3] = {ox, oy, oz};
  const jfli::DriftTables tb{chi, a_chi, n_chi, ga, g, n_g, da, dgfa, n_d};
  return cuda_status(jfli::healpix_paint_tiled_adjoint(disp, absolute, vel, weights, weight, d, box, obs, ntiles,
                                                       rotations, shifts, telephoto, rmin, rmax, t, gp_t, dbound, tb,
                                                       nside, scheme, map_bar, disp_bar, vel ? vel_bar : nullptr,
                                                       weights_bar, (cudaStream_t)stream),
                     err, errlen, "jfli_healpix_paint_tiled_adjoint");
}

int jfli_replica_positions(void* stream, const float* disp, int absolute, const float* vel, float lx, float ly,
                           float lz, float ox, float oy, float oz, const signed char* rotation, const float* shift,
                           int telephoto, float t, float gp_t, const float* chi, const float* a_chi, int n_chi,
                           const float* ga, const float* g, int n_g, const float* da, const float* dgfa, int n_d,
                           float* out, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(out);
  CHECK_PTR(rotation);
  CHECK_PTR(shift);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  int used = 0;
  for (int r = 0; r < 3; ++r) {
    int nnz = 0;
    for (int c = 0; c < 3; ++c) {
      const int m = rotation[3 * r + c];
      if (m == 0) continue;
      if ((m != 1 && m != -1) || (used & (1 << c)))
        return fail(err, errlen, JFLI_EINVAL, "rotation is not a signed permutation matrix");
      used |= 1 << c;
      ++nnz;
    }
    if (nnz != 1) return fail(err, errlen, JFLI_EINVAL, "rotation is not a signed permutation matrix");
  }
  if (vel) {
    CHECK_PTR(chi);
    CHECK_PTR(a_chi);
    CHECK_PTR(ga);
    CHECK_PTR(g);
    CHECK_PTR(da);
    CHECK_PTR(dgfa);
    if (n_chi < 2 || n_g < 2 || n_d < 2) return fail(err, errlen, JFLI_EINVAL, "tables need at least 2 entries");
    if (!(t > 0)) return fail(err, errlen, JFLI_EINVAL, "scale factor must be positive");
  }
  const MeshDims d{nx, ny, nz, batch};
  const float box[3] = {lx, ly, lz}, obs[3] = {ox, oy, oz};
  const jfli::DriftTables tb{chi, a_chi, n_chi, ga, g, n_g, da, dgfa, n_d};
  return cuda_status(jfli::replica_positions(disp, absolute, vel, d, box, obs, rotation, shift, telephoto, t, gp_t, tb,
                                             out, (cudaStream_t)stream),
                     err, errlen, "jfli_replica_positions");
}

int jfli_paint_flat(void* stream, const float* disp, int absolute, const float* weights, float weight, float zlo,
                    float zhi, int npx, int npy, float* map, int accumulate, int nx, int ny, int nz, int batch,
                    char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(map);
  if (npx < 1 || npy < 1 || (long long)npx * npy > (1LL << 30))
    return fail(err, errlen, JFLI_EINVAL, "flat-sky map (%d, %d) outside [1, 2^30] pixels", npx, npy);
  const MeshDims d{nx, ny, nz, batch};
  cudaStream_t s = (cudaStream_t)stream;
  if (!accumulate) {
    cudaError_t e = cudaMemsetAsync(map, 0, sizeof(float) * (size_t)npx * npy * batch, s);
    if (e != cudaSuccess) return cuda_status(e, err, errlen, "jfli_paint_flat memset");
  }
  return cuda_status(jfli::paint_flat(disp, absolute, weights, weight, d, npx, npy, zlo, zhi, map, s), err, errlen,
                     "jfli_paint_flat");
}

int jfli_paint_flat_adjoint(void* stream, const float* disp, int absolute, float weight, float zlo, float zhi, int npx,
                            int npy, const float* map_bar, float* pos_bar, int nx, int ny, int nz, int batch, char* err,
                            size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(map_bar);
  CHECK_PTR(pos_bar);
  if (npx < 1 || npy < 1 || (long long)npx * npy > (1LL << 30))
    return fail(err, errlen, JFLI_EINVAL, "flat-sky map (%d, %d) outside [1, 2^30] pixels", npx, npy);
  const MeshDims d{nx, ny, nz, batch};
  return cuda_status(jfli::paint_flat_adjoint(disp, absolute, weight, d, npx, npy, zlo, zhi, map_bar, pos_bar,
                                              (cudaStream_t)stream),
                     err, errlen, "jfli_paint_flat_adjoint");
}

static bool flat_fft_supported(int npx, int npy) {
  return npy % 2 == 0 && npy >= 4 && jfli::fft_axis_supported(npx) && jfli::fft_axis_supported(npy / 2);
}

size_t jfli_flat_cl_workspace_bytes(int npx, int npy, int batch, int nedges, int cross) {
  if (npx < 1 || npy < 2 || batch < 1 || nedges < 1) return 0;
  const size_t spec = align256(sizeof(float) * 2 * (size_t)npx * (npy / 2 + 1) * batch);
  return spec * (cross ? 2 : 1) +
         align256(sizeof(double) * 3 * (size_t)(nedges + 1) * jfli::flat_cl_ctas(npx, npy) * batch);
}

int jfli_flat_cl(void* stream, const float* map1, const float* map2, int npx, int npy, int batch, float dnx,
                 float dny, const float* ell_edges, int nedges, double* out, void* workspace, size_t workspace_bytes,
                 char* err, size_t errlen) {
  CHECK_PTR(map1);
  CHECK_PTR(ell_edges);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  if (batch < 1) return fail(err, errlen, JFLI_EINVAL, "batch must be >= 1");
  if (!flat_fft_supported(npx, npy))
    return fail(err, errlen, JFLI_EUNSUPPORTED,
                "flat-sky map (%d, %d) unsupported: npx must be 2^a 3^b <= 4096, npy even with npy/2 2^a 3^b", npx,
                npy);
  if (nedges < 1 || nedges > 1024) return fail(err, errlen, JFLI_EINVAL, "nedges %d outside [1, 1024]", nedges);
  if (!(dnx > 0 && dny > 0)) return fail(err, errlen, JFLI_EINVAL, "n * pixel size must be positive");
  const size_t need = jfli_flat_cl_workspace_bytes(npx, npy, batch, nedges, map2 != nullptr);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  const size_t spec = align256(sizeof(float) * 2 * (size_t)npx * (npy / 2 + 1) * batch);
  float2* s1 = (float2*)workspace;
  float2* s2 = map2 ? (float2*)((char*)workspace + spec) : nullptr;
  double* partials = (double*)((char*)workspace + spec * (map2 ? 2 : 1));
  return cuda_status(jfli::flat_cl(map1, map2, npx, npy, batch, dnx, dny, ell_edges, nedges, s1, s2, partials, out,
                                   (cudaStream_t)stream),
                     err, errlen, "jfli_flat_cl");
}

// P(k) for callers that cannot allocate device memory: the same sums as
// jfli_power_spectrum, with the half spectrum and the histogram partials kept in a
// fixed device array inside the library instead of a caller workspace. The array is
// shared by all calls on a device and holds the previous call's data; calls that
// overlap on the GPU (different streams, or host threads) race on it.
int jfli_power_spectrum_noalloc(void* stream, const float* mesh, const float* kedges, int nedges, float lx, float ly,
                                float lz, double* out, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(mesh);
  CHECK_PTR(kedges);
  CHECK_PTR(out);
  if (nedges < 1 || nedges > 2048) return fail(err, errlen, JFLI_EINVAL, "nedges %d outside [1, 2048]", nedges);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  const size_t spec = spec_bytes(d);
  const size_t partials = align256((size_t)jfli::noalloc_pk_ctas(d) * batch * 3 * (nedges + 1) * sizeof(double));
  const size_t cap = jfli::noalloc_scratch_bytes();
  if (spec + partials > cap)
    return fail(err, errlen, JFLI_EUNSUPPORTED,
                "mesh (%d, %d, %d) x batch %d with %d edges needs %zu bytes of scratch; the built-in scratch holds "
                "%zu bytes (up to a 128^3 mesh); use jfli_power_spectrum with a workspace",
                nx, ny, nz, batch, nedges, spec + partials, cap);
  void* base = nullptr;
  cudaError_t e = jfli::noalloc_scratch(&base);
  if (e != cudaSuccess) return cuda_status(e, err, errlen, "jfli_power_spectrum_noalloc scratch address");
  cudaStream_t s = (cudaStream_t)stream;
  const float box[3] = {lx, ly, lz};
  const float norm = 1.0f / ((float)nx * (float)ny * (float)nz);
  float2* specp = (float2*)base;
  double* part = (double*)((char*)base + spec);
  e = jfli::power_partials_noalloc(mesh, specp, part, d, kedges, nedges, box, norm, s);
  if (e == cudaSuccess) e = jfli::power_finalize(part, jfli::noalloc_pk_ctas(d), nedges + 1, out, batch, s);
  return cuda_status(e, err, errlen, "jfli_power_spectrum_noalloc");
}

int jfli_lightcone_drift(void* stream, const float* disp, const float* vel, float* out, float lx, float ly, float lz,
                         float ox, float oy, float oz, float t, float gp_t, const float* chi, const float* a_chi,
                         int n_chi, const float* ga, const float* g, int n_g, const float* da, const float* dgfa,
                         int n_d, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(vel);
  CHECK_PTR(out);
  CHECK_PTR(chi);
  CHECK_PTR(a_chi);
  CHECK_PTR(ga);
  CHECK_PTR(g);
  CHECK_PTR(da);
  CHECK_PTR(dgfa);
  if (n_chi < 2 || n_g < 2 || n_d < 2) return fail(err, errlen, JFLI_EINVAL, "tables need at least 2 entries");
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  if (!(t > 0)) return fail(err, errlen, JFLI_EINVAL, "scale factor must be positive");
  const MeshDims d{nx, ny, nz, batch};
  const float box[3] = {lx, ly, lz}, obs[3] = {ox, oy, oz};
  return cuda_status(jfli::lightcone_drift(disp, vel, out, box, obs, t, gp_t, chi, a_chi, n_chi, ga, g, n_g, da, dgfa,
                                           n_d, d, (cudaStream_t)stream),
                     err, errlen, "jfli_lightcone_drift");
}

size_t jfli_born_workspace_bytes(int nplanes, long long npix) {
  if (nplanes <= 0 || npix <= 0) return 0;
  return align256(sizeof(double) * (size_t)nplanes * jfli::born_ctas(npix)) + align256(sizeof(float) * nplanes);
}

int jfli_born(void* stream, const float* maps, int nplanes, long long npix, const float* weights, int nsrc,
              float* out, void* workspace, size_t workspace_bytes, char* err, size_t errlen) {
  CHECK_PTR(maps);
  CHECK_PTR(weights);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  if (nplanes < 1 || nplanes > 256) return fail(err, errlen, JFLI_EINVAL, "nplanes %d outside [1, 256]", nplanes);
  if (nsrc < 1 || nsrc > 32) return fail(err, errlen, JFLI_EINVAL, "nsrc %d outside [1, 32]", nsrc);
  if (npix < 1) return fail(err, errlen, JFLI_EINVAL, "npix must be positive");
  const size_t need = jfli_born_workspace_bytes(nplanes, npix);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  double* partials = (double*)workspace;
  float* mean = (float*)((char*)workspace + align256(sizeof(double) * (size_t)nplanes * jfli::born_ctas(npix)));
  return cuda_status(
      jfli::born_convergence(maps, nplanes, npix, weights, nsrc, out, partials, mean, (cudaStream_t)stream), err,
      errlen, "jfli_born");
}

size_t jfli_born_adjoint_workspace_bytes(int nplanes, long long npix) {
  return jfli_born_workspace_bytes(nplanes, npix) + align256(sizeof(float) * (nplanes > 0 ? nplanes : 0));
}

int jfli_born_adjoint(void* stream, const float* maps, int nplanes, long long npix, const float* weights, int nsrc,
                      const float* kappa_bar, float* maps_bar, void* workspace, size_t workspace_bytes, char* err,
                      size_t errlen) {
  CHECK_PTR(maps);
  CHECK_PTR(weights);
  CHECK_PTR(kappa_bar);
  CHECK_PTR(maps_bar);
  CHECK_PTR(workspace);
  if (nplanes < 1 || nplanes > 256) return fail(err, errlen, JFLI_EINVAL, "nplanes %d outside [1, 256]", nplanes);
  if (nsrc < 1 || nsrc > 32) return fail(err, errlen, JFLI_EINVAL, "nsrc %d outside [1, 32]", nsrc);
  if (npix < 1) return fail(err, errlen, JFLI_EINVAL, "npix must be positive");
  const size_t need = jfli_born_adjoint_workspace_bytes(nplanes, npix);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  double* partials = (double*)workspace;
  float* mean = (float*)((char*)workspace + align256(sizeof(double) * (size_t)nplanes * jfli::born_ctas(npix)));
  float* c = (float*)((char*)workspace + jfli_born_workspace_bytes(nplanes, npix));
  return cuda_status(jfli::born_convergence_adjoint(maps, nplanes, npix, weights, nsrc, kappa_bar, maps_bar,
                                                    partials, mean, c, (cudaStream_t)stream),
                     err, errlen, "jfli_born_adjoint");
}

int jfli_born_flat(void* stream, const float* maps, int nplanes, int n0, int n1, const float* weights, int nsrc,
                   const float* s0, const float* s1, float* out, void* workspace, size_t workspace_bytes, char* err,
                   size_t errlen) {
  CHECK_PTR(maps);
  CHECK_PTR(weights);
  CHECK_PTR(s0);
  CHECK_PTR(s1);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  if (nplanes < 1 || nplanes > 256) return fail(err, errlen, JFLI_EINVAL, "nplanes %d outside [1, 256]", nplanes);
  if (nsrc < 1 || nsrc > 32) return fail(err, errlen, JFLI_EINVAL, "nsrc %d outside [1, 32]", nsrc);
  if (n0 < 1 || n1 < 1) return fail(err, errlen, JFLI_EINVAL, "plane shape must be positive");
  const long long npix = (long long)n0 * n1;
  const size_t need = jfli_born_workspace_bytes(nplanes, npix);
  if (workspace_bytes < need)
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, need);
  double* partials = (double*)workspace;
  float* mean = (float*)((char*)workspace + align256(sizeof(double) * (size_t)nplanes * jfli::born_ctas(npix)));
  return cuda_status(jfli::born_flat(maps, nplanes, n0, n1, weights, nsrc, s0, s1, out, partials, mean,
                                     (cudaStream_t)stream),
                     err, errlen, "jfli_born_flat");
}

int jfli_sht_map2alm(void* stream, const double* F, const double* z, int nrings, int lmax, double weight,
                     double* alm, char* err, size_t errlen) {
  CHECK_PTR(F);
  CHECK_PTR(z);
  CHECK_PTR(alm);
  if (nrings < 1 || nrings > 65535) return fail(err, errlen, JFLI_EINVAL, "nrings %d outside [1, 65535]", nrings);
  if (lmax < 0 || lmax > 8191) return fail(err, errlen, JFLI_EINVAL, "lmax %d outside [0, 8191]", lmax);
  return cuda_status(jfli::sht_analysis(F, z, nrings, lmax, weight, alm, (cudaStream_t)stream), err, errlen,
                     "jfli_sht_map2alm");
}

int jfli_sht_ring_analysis(void* stream, const double* map, int nside, int lmax, double* F, char* err,
                           size_t errlen) {
  CHECK_PTR(map);
  CHECK_PTR(F);
  if (nside < 1 || nside > 4096) return fail(err, errlen, JFLI_EINVAL, "nside %d outside [1, 4096]", nside);
  if (lmax < 0 || lmax > 8191) return fail(err, errlen, JFLI_EINVAL, "lmax %d outside [0, 8191]", lmax);
  return cuda_status(jfli::sht_ring_analysis(map, nside, lmax, F, (cudaStream_t)stream), err, errlen,
                     "jfli_sht_ring_analysis");
}

int jfli_sht_ring_synthesis(void* stream, const double* G, int nside, int lmax, double* map, char* err,
                            size_t errlen) {
  CHECK_PTR(G);
  CHECK_PTR(map);
  if (nside < 1 || nside > 4096) return fail(err, errlen, JFLI_EINVAL, "nside %d outside [1, 4096]", nside);
  if (lmax < 0 || lmax > 8191) return fail(err, errlen, JFLI_EINVAL, "lmax %d outside [0, 8191]", lmax);
  return cuda_status(jfli::sht_ring_synthesis(G, nside, lmax, map, (cudaStream_t)stream), err, errlen,
                     "jfli_sht_ring_synthesis");
}

int jfli_sht_alm2map(void* stream, const double* alm, const double* z, int nrings, int lmax, double* G, char* err,
                     size_t errlen) {
  CHECK_PTR(alm);
  CHECK_PTR(z);
  CHECK_PTR(G);
  if (nrings < 1 || nrings > 65535) return fail(err, errlen, JFLI_EINVAL, "nrings %d outside [1, 65535]", nrings);
  if (lmax < 0 || lmax > 8191) return fail(err, errlen, JFLI_EINVAL, "lmax %d outside [0, 8191]", lmax);
  return cuda_status(jfli::sht_synthesis(alm, z, nrings, lmax, G, (cudaStream_t)stream), err, errlen,
                     "jfli_sht_alm2map");
}

int jfli_zero(void* stream, float* data, long long n, char* err, size_t errlen) {
  CHECK_PTR(data);
  if (n < 0) return fail(err, errlen, JFLI_EINVAL, "n must be >= 0");
  return cuda_status(jfli::zero_floats(data, n, (cudaStream_t)stream), err, errlen, "jfli_zero");
}

int jfli_set_fft_x_pass(int mode, char* err, size_t errlen) {
  if (mode != 0 && mode != 1) return fail(err, errlen, JFLI_EINVAL, "x pass mode %d is not 0 or 1", mode);
  jfli::set_x_pass_mode(mode);
  return JFLI_OK;
}

int jfli_device_status(unsigned* status, int reset, char* err, size_t errlen) {
  CHECK_PTR(status);
  return cuda_status(jfli::device_status(status, reset != 0), err, errlen, "jfli_device_status");
}

int jfli_sht_alm2cl(void* stream, const double* alm1, const double* alm2, int lmax, double* cl, char* err,
                    size_t errlen) {
  CHECK_PTR(alm1);
  CHECK_PTR(cl);
  if (lmax < 0 || lmax > 8191) return fail(err, errlen, JFLI_EINVAL, "lmax %d outside [0, 8191]", lmax);
  return cuda_status(jfli::sht_alm2cl(alm1, alm2, lmax, cl, (cudaStream_t)stream), err, errlen, "jfli_sht_alm2cl");
}

// ---- reversible KKD loop and its reverse sweep -------------------------------------
namespace {
struct KkdWs {
  float2* spec;
  float *pot, *rho, *rho_bar, *div, *force, *ubar;
  double* partials;
};

// ubar is one float4 mesh (the cotangent paint takes one vector atomic per corner)
size_t kkd_ws_bytes(const MeshDims& d) {
  return spec_bytes(d) + 4 * mesh_bytes(d) + align256(sizeof(float) * 4 * (size_t)d.cells() * d.batch) +
         align256(sizeof(float) * 4 * (size_t)d.cells() * d.batch) +
         align256(sizeof(double) * jfli::adjoint_partials_count(d));
}

KkdWs kkd_ws(void* w, const MeshDims& d) {
  char* p = (char*)w;
  KkdWs k;
  k.spec = (float2*)p;
  p += spec_bytes(d);
  k.pot = (float*)p;
  p += mesh_bytes(d);
  k.rho = (float*)p;
  p += mesh_bytes(d);
  k.rho_bar = (float*)p;
  p += mesh_bytes(d);
  k.div = (float*)p;
  p += mesh_bytes(d);
  k.force = (float*)p;
  p += align256(sizeof(float) * 4 * (size_t)d.cells() * d.batch);
  k.ubar = (float*)p;
  p += align256(sizeof(float) * 4 * (size_t)d.cells() * d.batch);
  k.partials = (double*)p;
  return k;
}

// SharpeningKernel in the reversible step: per-step velocity boost factors alpha / drift and
// the PGD scales; boosts == nullptr is the plain step. With boosts, step i's force is the
// combined one, kicks[i] F + boosts[i] F_pgd at the same positions, applied with factor 1.
struct Sharpen {
  const float* boosts = nullptr;
  float kl = 0.f, ks = 1.f;
};

// The potential whose force kicks step i (the mean 1 of a painted density; 0 for the
// divergence of a cotangent mesh, whose solve is the same symmetric operator).
cudaError_t step_potential(const float* src, float2* spec, float* pot, const MeshDims& d, float mean,
                           const float* kicks, int i, const Sharpen& sh, cudaStream_t s) {
  if (sh.boosts) return jfli::mixed_pgd_potential(src, spec, pot, d, mean, sh.kl, sh.ks, kicks[i], sh.boosts[i], 1.0f, s);
  return jfli::poisson_potential(src, spec, pot, d, mean, 1.0f, s);
}

// the factor the force mesh of step i is applied with
float step_kick(const float* kicks, int i, const Sharpen& sh) { return sh.boosts ? 1.0f : kicks[i]; }

// density of the current positions -> potential of step i (into pot) -> force mesh (in ws.force)
cudaError_t kkd_force(float* disp, float* vel, float* rho, const KkdWs& w, float* pot, const MeshDims& d,
                      cudaStream_t s, const float* kicks, int i, const Sharpen& sh) {
  cudaError_t e = cudaMemsetAsync(rho, 0, (size_t)d.cells() * d.batch * sizeof(float), s);
  if (e == cudaSuccess) e = jfli::kick_drift_paint(disp, vel, nullptr, 0.f, 0.f, JFLI_STEP_PAINT, 1.0f, rho, d, s);
  if (e == cudaSuccess) e = step_potential(rho, w.spec, pot, d, 1.0f, kicks, i, sh, s);
  if (e == cudaSuccess) e = jfli::force_mesh(pot, w.force, 1.0f, d, s);
  return e;
}

// The loop of jfli_kkd_run; with pots (nsteps potentials [step][batch][cells]) the
// potential whose force kicks step i is written to pots[i] instead of the workspace.
int kkd_run_impl(void* stream, float* disp, float* vel, const float* kicks, const float* drifts, int nsteps,
                 float* rho, float* pots, void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch,
                 char* err, size_t errlen, const char* name, const Sharpen& sh = Sharpen()) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(disp);
  CHECK_PTR(vel);
  CHECK_PTR(kicks);
  CHECK_PTR(drifts);
  CHECK_PTR(rho);
  CHECK_PTR(workspace);
  CHECK_ALIGN16(workspace);
  if (nsteps < 0) return fail(err, errlen, JFLI_EINVAL, "nsteps must be >= 0");
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < kkd_ws_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, kkd_ws_bytes(d));
  cudaStream_t s = (cudaStream_t)stream;
  const KkdWs w = kkd_ws(workspace, d);
  const size_t per = (size_t)d.cells() * batch;
  auto pot_of = [&](int i) { return pots ? pots + (size_t)i * per : w.pot; };
  // rho is cleared right before each paint (zeroed lines still in L2 when the deposits come);
  // the last step's paint stays in rho (the density of the final positions)
  cudaError_t e = nsteps > 0 ? kkd_force(disp, vel, rho, w, pot_of(0), d, s, kicks, 0, sh)
                             : kkd_force(disp, vel, rho, w, pot_of(0), d, s, kicks, 0, Sharpen());
  for (int i = 0; i < nsteps && e == cudaSuccess; ++i) {
    e = jfli::zero_floats(rho, d.cells() * batch, s);
    if (e == cudaSuccess)
      e = jfli::kick_drift_paint(disp, vel, w.force, step_kick(kicks, i, sh), drifts[i],
                                 JFLI_STEP_KICK | JFLI_STEP_DRIFT | JFLI_STEP_PAINT, 1.0f, rho, d, s);
    if (e == cudaSuccess && i + 1 < nsteps) e = step_potential(rho, w.spec, pot_of(i + 1), d, 1.0f, kicks, i + 1, sh, s);
    if (e == cudaSuccess && i + 1 < nsteps) e = jfli::force_mesh(pot_of(i + 1), w.force, 1.0f, d, s);
  }
  return cuda_status(e, err, errlen, name);
}

// The reverse sweep of jfli_kkd_adjoint. Without pots each step un-drifts and paints the
// previous positions and solves for their force; with pots the force mesh is rebuilt from
// the stored potential and the un-drift happens inside the cotangent paint.
int kkd_adjoint_impl(void* stream, float* disp, float* vel, float* lam_x, float* lam_v, const float* kicks,
                     const float* drifts, int nsteps, const float* pots, double* sens, void* workspace,
                     size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen,
                     const char* name, const Sharpen& sh = Sharpen()) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(disp);
  CHECK_PTR(vel);
  CHECK_PTR(lam_x);
  CHECK_PTR(lam_v);
  CHECK_PTR(kicks);
  CHECK_PTR(drifts);
  CHECK_PTR(sens);
  CHECK_PTR(workspace);
  CHECK_ALIGN16(workspace);
  if (nsteps < 0) return fail(err, errlen, JFLI_EINVAL, "nsteps must be >= 0");
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < kkd_ws_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, kkd_ws_bytes(d));
  cudaStream_t s = (cudaStream_t)stream;
  const KkdWs w = kkd_ws(workspace, d);
  const size_t per = (size_t)d.cells() * batch;
  cudaError_t e = cudaSuccess;
  for (int i = nsteps - 1; i >= 0 && e == cudaSuccess; --i) {
    const float k = step_kick(kicks, i, sh), dr = drifts[i];
    if (pots) {
      // the force mesh of step i from its stored potential; un-drift in the paint below
      e = jfli::force_mesh(pots + (size_t)i * per, w.force, 1.0f, d, s);
    } else {
      // un-drift and paint the previous positions, force mesh there
      e = jfli::zero_floats(w.rho, d.cells() * batch, s);
      if (e == cudaSuccess)
        e = jfli::kick_drift_paint(disp, vel, nullptr, 0.f, -dr, JFLI_STEP_DRIFT | JFLI_STEP_PAINT, 1.0f, w.rho, d, s);
      if (e == cudaSuccess) e = step_potential(w.rho, w.spec, w.pot, d, 1.0f, kicks, i, sh, s);
      if (e == cudaSuccess) e = jfli::force_mesh(w.pot, w.force, 1.0f, d, s);
    }
    // un-kick, adjoint paint, dL/dk and dL/dd (with sharpening, dL/d of the combined force's
    // factor 1 in place of dL/dk)
    if (e == cudaSuccess)
      e = jfli::adjoint_unkick_paint(disp, vel, lam_x, lam_v, w.force, k, dr, w.ubar, w.partials, d, s, true,
                                     pots ? disp : nullptr);
    if (e == cudaSuccess) e = jfli::sum_adjoint_partials(w.partials, d, sens + 2ll * i * batch, s);
    // rho_bar = P(div ubar); lam_x += k grad R[rho_bar + lam_v . F]
    if (e == cudaSuccess) e = jfli::divergence_fd(w.ubar, 1.0f, nullptr, 0.0f, 2, 0, w.div, d, s);
    if (e == cudaSuccess) e = step_potential(w.div, w.spec, w.rho_bar, d, 0.0f, kicks, i, sh, s);
    if (e == cudaSuccess) e = jfli::adjoint_position(disp, lam_v, w.rho_bar, w.force, k, lam_x, d, s);
  }
  return cuda_status(e, err, errlen, name);
}
}  // namespace

size_t jfli_kkd_workspace_bytes(int nx, int ny, int nz, int batch) {
  return kkd_ws_bytes(MeshDims{nx, ny, nz, batch});
}

int jfli_kkd_run(void* stream, float* disp, float* vel, const float* kicks, const float* drifts, int nsteps,
                 float* rho, void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                 size_t errlen) {
  return kkd_run_impl(stream, disp, vel, kicks, drifts, nsteps, rho, nullptr, workspace, workspace_bytes, nx, ny, nz,
                      batch, err, errlen, "jfli_kkd_run");
}

int jfli_kkd_run_stored(void* stream, float* disp, float* vel, const float* kicks, const float* drifts, int nsteps,
                        float* rho, float* pots, void* workspace, size_t workspace_bytes, int nx, int ny, int nz,
                        int batch, char* err, size_t errlen) {
  CHECK_PTR(pots);
  return kkd_run_impl(stream, disp, vel, kicks, drifts, nsteps, rho, pots, workspace, workspace_bytes, nx, ny, nz,
                      batch, err, errlen, "jfli_kkd_run_stored");
}

int jfli_kkd_adjoint(void* stream, float* disp, float* vel, float* lam_x, float* lam_v, const float* kicks,
                     const float* drifts, int nsteps, double* sens, void* workspace, size_t workspace_bytes, int nx,
                     int ny, int nz, int batch, char* err, size_t errlen) {
  return kkd_adjoint_impl(stream, disp, vel, lam_x, lam_v, kicks, drifts, nsteps, nullptr, sens, workspace,
                          workspace_bytes, nx, ny, nz, batch, err, errlen, "jfli_kkd_adjoint");
}

int jfli_kkd_adjoint_stored(void* stream, float* disp, float* vel, float* lam_x, float* lam_v, const float* kicks,
                            const float* drifts, int nsteps, const float* pots, double* sens, void* workspace,
                            size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_PTR(pots);
  return kkd_adjoint_impl(stream, disp, vel, lam_x, lam_v, kicks, drifts, nsteps, pots, sens, workspace,
                          workspace_bytes, nx, ny, nz, batch, err, errlen, "jfli_kkd_adjoint_stored");
}

int jfli_kkd_run_sharpened(void* stream, float* disp, float* vel, const float* kicks, const float* drifts,
                           const float* boosts, float kl, float ks, int nsteps, float* rho, float* pots, void* workspace,
                           size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_PTR(boosts);
  if (!(kl >= 0.0f && ks > 0.0f)) return fail(err, errlen, JFLI_EINVAL, "PGD scales need kl >= 0 and ks > 0");
  Sharpen sh;
  sh.boosts = boosts;
  sh.kl = kl;
  sh.ks = ks;
  return kkd_run_impl(stream, disp, vel, kicks, drifts, nsteps, rho, pots, workspace, workspace_bytes, nx, ny, nz,
                      batch, err, errlen, "jfli_kkd_run_sharpened", sh);
}

int jfli_kkd_adjoint_sharpened(void* stream, float* disp, float* vel, float* lam_x, float* lam_v, const float* kicks,
                               const float* drifts, const float* boosts, float kl, float ks, int nsteps,
                               const float* pots, double* sens, void* workspace, size_t workspace_bytes, int nx,
                               int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_PTR(boosts);
  if (!(kl >= 0.0f && ks > 0.0f)) return fail(err, errlen, JFLI_EINVAL, "PGD scales need kl >= 0 and ks > 0");
  Sharpen sh;
  sh.boosts = boosts;
  sh.kl = kl;
  sh.ks = ks;
  return kkd_adjoint_impl(stream, disp, vel, lam_x, lam_v, kicks, drifts, nsteps, pots, sens, workspace,
                          workspace_bytes, nx, ny, nz, batch, err, errlen, "jfli_kkd_adjoint_sharpened", sh);
}

int jfli_sharpen_potential(void* stream, const float* rho, float rho_mean, float kick, float boost, float kl, float ks,
                           float* pot, void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch,
                           char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(rho);
  CHECK_PTR(pot);
  CHECK_PTR(workspace);
  CHECK_ALIGN16(workspace);
  if (!(kl >= 0.0f && ks > 0.0f)) return fail(err, errlen, JFLI_EINVAL, "PGD scales need kl >= 0 and ks > 0");
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < spec_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, spec_bytes(d));
  return cuda_status(jfli::mixed_pgd_potential(rho, (float2*)workspace, pot, d, rho_mean, kl, ks, kick, boost, 1.0f,
                                               (cudaStream_t)stream),
                     err, errlen, "jfli_sharpen_potential");
}

// ---- adjoints --------------------------------------------------------------------
size_t jfli_adjoint_partials_count(int nx, int ny, int nz, int batch) {
  return jfli::adjoint_partials_count(MeshDims{nx, ny, nz, batch});
}

int jfli_adjoint_unkick_paint(void* stream, const float* disp, float* vel, const float* lam_x, float* lam_v,
                              const float* force, float kick, float drift, float* ubar, double* partials,
                              size_t partials_count, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(vel);
  CHECK_PTR(lam_x);
  CHECK_PTR(lam_v);
  CHECK_PTR(force);
  CHECK_ALIGN16(force);
  CHECK_PTR(ubar);
  CHECK_PTR(partials);
  const MeshDims d{nx, ny, nz, batch};
  const size_t need = jfli::adjoint_partials_count(d);
  if (partials_count < need)
    return fail(err, errlen, JFLI_EINVAL, "partials hold %zu doubles, need %zu", partials_count, need);
  return cuda_status(jfli::adjoint_unkick_paint(disp, vel, lam_x, lam_v, force, kick, drift, ubar, partials, d,
                                                (cudaStream_t)stream),
                     err, errlen, "jfli_adjoint_unkick_paint");
}

size_t jfli_poisson_divergence_workspace_bytes(int nx, int ny, int nz, int batch) {
  const MeshDims d{nx, ny, nz, batch};
  return spec_bytes(d) + mesh_bytes(d);
}

int jfli_poisson_divergence(void* stream, const float* u, float alpha, const float* w, float beta, int aos, float scale,
                            float* out, void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch,
                            char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(u);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < jfli_poisson_divergence_workspace_bytes(nx, ny, nz, batch))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes,
                jfli_poisson_divergence_workspace_bytes(nx, ny, nz, batch));
  cudaStream_t s = (cudaStream_t)stream;
  float2* spec = (float2*)workspace;
  float* div = (float*)((char*)workspace + spec_bytes(d));
  cudaError_t e = jfli::divergence_fd(u, alpha, w, beta, aos ? 1 : 0, 0, div, d, s);
  if (e == cudaSuccess) e = jfli::poisson_potential(div, spec, out, d, 0.0f, scale, s);
  return cuda_status(e, err, errlen, "jfli_poisson_divergence");
}

int jfli_adjoint_position(void* stream, const float* disp, const float* u, const float* rho_bar, const float* force,
                          float scale, float* lam_x, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_PTR(disp);
  CHECK_PTR(lam_x);
  if ((u == nullptr) != (force == nullptr))
    return fail(err, errlen, JFLI_EINVAL, "u and force must be given together");
  if (force) CHECK_ALIGN16(force);
  if (rho_bar == nullptr && force == nullptr) return fail(err, errlen, JFLI_EINVAL, "nothing to read out");
  const MeshDims d{nx, ny, nz, batch};
  return cuda_status(jfli::adjoint_position(disp, u, rho_bar, force, scale, lam_x, d, (cudaStream_t)stream), err,
                     errlen, "jfli_adjoint_position");
}

int jfli_power_poles_adjoint(void* stream, const float* mesh, const float* kedges, const float* weights, int nedges,
                             const int* ells, int nell, int complex_weights, float lx, float ly, float lz,
                             float losx, float losy, float losz, float* out, void* workspace, size_t workspace_bytes,
                             int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(mesh);
  CHECK_PTR(kedges);
  CHECK_PTR(weights);
  CHECK_PTR(ells);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  // 8: the multipole slots of the adjoint operator (kMaxAdjPoles)
  if (nell < 1 || nell > 8) return fail(err, errlen, JFLI_EINVAL, "nell %d outside [1, 8]", nell);
  const int cplx = complex_weights ? 1 : 0;
  if (nedges < 1 || nedges + (1 + cplx) * nell * (nedges + 1) > 2 * 2048 + 1)
    return fail(err, errlen, JFLI_EINVAL, "nedges %d with %d multipoles exceeds the weight table", nedges, nell);
  for (int e = 0; e < nell; ++e)
    if (ells[e] < 0 || ells[e] > 16) return fail(err, errlen, JFLI_EINVAL, "multipole %d outside [0, 16]", ells[e]);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const double ln = std::sqrt((double)losx * losx + (double)losy * losy + (double)losz * losz);
  if (!(ln > 0)) return fail(err, errlen, JFLI_EINVAL, "the line of sight must be nonzero");
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < spec_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, spec_bytes(d));
  const float box[3] = {lx, ly, lz};
  const float los[3] = {(float)(losx / ln), (float)(losy / ln), (float)(losz / ln)};
  return cuda_status(jfli::power_poles_adjoint(mesh, (float2*)workspace, out, d, kedges, weights, nedges, ells, nell,
                                               box, los, cplx, (cudaStream_t)stream),
                     err, errlen, "jfli_power_poles_adjoint");
}

int jfli_power_spectrum_adjoint(void* stream, const float* mesh, const float* kedges, const float* weights,
                                int nedges, float lx, float ly, float lz, float* out, void* workspace,
                                size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(mesh);
  CHECK_PTR(kedges);
  CHECK_PTR(weights);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  if (nedges < 1 || nedges > 2048) return fail(err, errlen, JFLI_EINVAL, "nedges %d outside [1, 2048]", nedges);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < spec_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, spec_bytes(d));
  const float box[3] = {lx, ly, lz};
  return cuda_status(jfli::power_adjoint(mesh, (float2*)workspace, out, d, kedges, weights, nedges, box,
                                         (cudaStream_t)stream),
                     err, errlen, "jfli_power_spectrum_adjoint");
}

size_t jfli_lpt_adjoint_workspace_bytes(int nx, int ny, int nz, int batch) {
  const MeshDims d{nx, ny, nz, batch};
  return spec_bytes(d) + 9 * mesh_bytes(d);
}

int jfli_lpt_adjoint(void* stream, const float* ic, int order, float c1x, float c2x, float c1p, float c2p,
                     const float* lam_x, const float* lam_v, float* out, void* workspace, size_t workspace_bytes,
                     int nx, int ny, int nz, int batch, char* err, size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_STENCIL(nx, ny, nz);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(ic);
  CHECK_PTR(lam_x);
  CHECK_PTR(lam_v);
  CHECK_PTR(out);
  CHECK_PTR(workspace);
  if (order != 1 && order != 2) return fail(err, errlen, JFLI_EINVAL, "LPT order must be 1 or 2, got %d", order);
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < jfli_lpt_adjoint_workspace_bytes(nx, ny, nz, batch))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes,
                jfli_lpt_adjoint_workspace_bytes(nx, ny, nz, batch));
  cudaStream_t s = (cudaStream_t)stream;
  char* w = (char*)workspace;
  float2* spec = (float2*)w;
  float* phi1 = (float*)(w + spec_bytes(d));
  float* sbar = (float*)(w + spec_bytes(d) + mesh_bytes(d));
  float* acc = (float*)(w + spec_bytes(d) + 2 * mesh_bytes(d));
  float* q = (float*)(w + spec_bytes(d) + 3 * mesh_bytes(d));
  // dx = c1x F1 + c2x F2, p = c1p c1x F1 + c2p c2x F2 with F_i = -D P s_i (s_1 = ic,
  // s_2 = delta2(P ic)); (-D P)^T = P div, so dL/ds_i = P div(ubar_i) with
  // ubar_1 = c1x lam_x + c1p c1x lam_v, ubar_2 = c2x lam_x + c2p c2x lam_v.
  cudaError_t e = jfli::divergence_fd(lam_x, c1x, lam_v, c1p * c1x, 1, 0, acc, d, s);
  if (e == cudaSuccess && order == 2) {
    e = jfli::poisson_potential(ic, spec, phi1, d, 0.0f, 1.0f, s);
    if (e == cudaSuccess) e = jfli::divergence_fd(lam_x, c2x, lam_v, c2p * c2x, 1, 0, sbar, d, s);
    if (e == cudaSuccess) e = jfli::poisson_potential(sbar, spec, sbar, d, 0.0f, 1.0f, s);
    // dL/dphi1 accumulated into acc, then the common P: dL/dic = P(div ubar_1 + dL/dphi1)
    if (e == cudaSuccess) e = jfli::lpt2_source_adjoint(phi1, sbar, q, acc, 1, d, s);
  }
  if (e == cudaSuccess) e = jfli::poisson_potential(acc, spec, out, d, 0.0f, 1.0f, s);
  return cuda_status(e, err, errlen, "jfli_lpt_adjoint");
}

int jfli_ic_filter_tangent(void* stream, const float* noise, float* out, const float* ktab, const float* ptab,
                           const float* dptab, int ntab, float lx, float ly, float lz, int zero_mode_one,
                           void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                           size_t errlen) {
  CHECK_DIMS(nx, ny, nz, batch);
  CHECK_FFT(nx, ny, nz);
  CHECK_PTR(noise);
  CHECK_PTR(out);
  CHECK_PTR(ktab);
  CHECK_PTR(ptab);
  CHECK_PTR(dptab);
  CHECK_PTR(workspace);
  if (ntab < 2 || ntab > 4096) return fail(err, errlen, JFLI_EINVAL, "table length %d outside [2, 4096]", ntab);
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(err, errlen, JFLI_EINVAL, "box sizes must be positive");
  const MeshDims d{nx, ny, nz, batch};
  if (workspace_bytes < spec_bytes(d))
    return fail(err, errlen, JFLI_EINVAL, "workspace too small: %zu < %zu bytes", workspace_bytes, spec_bytes(d));
  const float box[3] = {lx, ly, lz};
  return cuda_status(jfli::ic_filter(noise, (float2*)workspace, out, d, ktab, ptab, ntab, box, zero_mode_one,
                                     (cudaStream_t)stream, dptab),
                     err, errlen, "jfli_ic_filter_tangent");
}

}  // extern "C"
