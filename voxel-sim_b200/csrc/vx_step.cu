// vx_step.cu — the fixed step of the elastic path on the device: the explicit
// prediction and the velocity update of solver::step_with_axis_targets_and_loads
// (src/solver.rs:438-700) around the rotation fit and corotational passes.
#include <cmath>

#include "vx_device.cuh"
#include "vx_kernels.h"

namespace vx {

// Substep prediction (src/solver.rs:490-517): previous = x; for free REVs
// v += g h, targeted axes get v = 0, drift = v, x += v h; then every targeted
// axis is set to its target; predicted = x. Kinematic REVs keep x and v.
__global__ void k_predict(uint32_t n, double* __restrict__ pos, double* __restrict__ vel, double* __restrict__ prev,
                          double* __restrict__ drift, double* __restrict__ pred, const uint8_t* __restrict__ kin,
                          const uint8_t* __restrict__ tmask, const double* __restrict__ target, double3 g, double h,
                          const uint8_t* __restrict__ tile_on) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !tile_active(tile_on, i)) return;
    const uint8_t tm = tmask[i];
    const bool free_rev = kin[i] == 0;
    const double ga[3] = {g.x, g.y, g.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const size_t t = (size_t)a * n + i;
        double x = pos[t];
        prev[t] = x;
        double d = 0.0;
        if (free_rev) {
            double v = vel[t] + ga[a] * h;
            if ((tm >> a) & 1) v = 0.0;
            vel[t] = v;
            d = v;
            x += v * h;
        }
        if ((tm >> a) & 1) x = target[t];
        drift[t] = d;
        pos[t] = x;
        pred[t] = x;
    }
}

// Velocity update after the passes (src/solver.rs:667-681): targeted axes
// (x - previous) / h, other axes drift + (x - predicted) / h; kinematic REVs
// are left alone.
__global__ void k_velocity(uint32_t n, const double* __restrict__ pos, double* __restrict__ vel,
                           const double* __restrict__ prev, const double* __restrict__ drift,
                           const double* __restrict__ pred, const uint8_t* __restrict__ kin,
                           const uint8_t* __restrict__ tmask, double h, const uint8_t* __restrict__ tile_on) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !tile_active(tile_on, i) || kin[i]) return;
    const uint8_t tm = tmask[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const size_t t = (size_t)a * n + i;
        vel[t] = ((tm >> a) & 1) ? (pos[t] - prev[t]) / h : drift[t] + (pos[t] - pred[t]) / h;
    }
}

// Indexed velocity writes: op 0 sets, op 1 adds; targeted axes stay zero
// (set_velocity / apply_impulse, src/solver.rs:207-255).
__global__ void k_velocity_update(uint32_t n, uint32_t count, const uint32_t* __restrict__ index,
                                  const double* __restrict__ value, int32_t op, double* __restrict__ vel,
                                  const uint8_t* __restrict__ tmask) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint32_t i = index[k];
    if (i >= n) return;
    const uint8_t tm = tmask[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const size_t t = (size_t)a * n + i;
        const double v = op == 1 ? vel[t] + value[3 * (size_t)k + a] : value[3 * (size_t)k + a];
        vel[t] = ((tm >> a) & 1) ? 0.0 : v;
    }
}

// Indexed gather / scatter of a [3][n] field (AoS values, 3 per entry).
__global__ void k_gather3(uint32_t n, uint32_t count, const uint32_t* __restrict__ index,
                          const double* __restrict__ field, double* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint32_t i = index[k];
    if (i >= n) return;
#pragma unroll
    for (int a = 0; a < 3; ++a) out[3 * (size_t)k + a] = field[(size_t)a * n + i];
}
__global__ void k_scatter3(uint32_t n, uint32_t count, const uint32_t* __restrict__ index,
                           const double* __restrict__ value, double* __restrict__ field) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint32_t i = index[k];
    if (i >= n) return;
#pragma unroll
    for (int a = 0; a < 3; ++a) field[(size_t)a * n + i] = value[3 * (size_t)k + a];
}

cudaError_t launch_gather3(vx_scene* s, uint32_t count, const uint32_t* d_index, const double* field, double* d_out) {
    if (count == 0) return cudaSuccess;
    k_gather3<<<(count + 255) / 256, 256, 0, s->stream>>>(s->n, count, d_index, field, d_out);
    return cudaGetLastError();
}
cudaError_t launch_scatter3(vx_scene* s, uint32_t count, const uint32_t* d_index, const double* d_value,
                            double* field) {
    if (count == 0) return cudaSuccess;
    k_scatter3<<<(count + 255) / 256, 256, 0, s->stream>>>(s->n, count, d_index, d_value, field);
    return cudaGetLastError();
}

// Targets that move (mask bit VX_TARGET_MOVING) advance by their slot's delta
// on their targeted axes; delta[3 * slot + a].
__global__ void k_advance_targets(uint32_t n, const uint8_t* __restrict__ tmask, double* __restrict__ target,
                                  const double* __restrict__ delta, const uint8_t* __restrict__ tile_on,
                                  const uint32_t* __restrict__ tile_scene) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !tile_active(tile_on, i)) return;
    const uint8_t tm = tmask[i];
    if (!(tm & VX_TARGET_MOVING)) return;
    const uint32_t slot = tile_scene ? tile_scene[i >> 8] : 0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if ((tm >> a) & 1) target[(size_t)a * n + i] += delta[3 * (size_t)slot + a];
}

cudaError_t launch_advance_targets(vx_scene* s, const double* d_delta) {
    if (s->n == 0) return cudaSuccess;
    k_advance_targets<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->tmask, s->target, d_delta, s->tile_on,
                                                                 s->tile_scene);
    return cudaGetLastError();
}

cudaError_t launch_predict(vx_scene* s, const double* gravity, double h) {
    if (s->n == 0) return cudaSuccess;
    k_predict<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->pos, s->vel, s->prev, s->drift, s->pred, s->kin,
                                                         s->tmask, s->target,
                                                         make_double3(gravity[0], gravity[1], gravity[2]), h,
                                                         s->tile_on);
    return cudaGetLastError();
}

// rest[a][first + t] = pos[a][first + t] in f32, t < count, every axis
__global__ void k_rest_positions(uint32_t n, size_t first, size_t count, const double* __restrict__ pos,
                                 float* __restrict__ rest) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= 3 * count) return;
    const size_t k = (t / count) * n + first + t % count;
    rest[k] = (float)pos[k];
}

// Scene::rest_positions: the creation positions in f32 (src/scene.rs:520-522)
cudaError_t launch_rest_range(vx_scene* s, size_t first, size_t count) {
    if (count == 0) return cudaSuccess;
    k_rest_positions<<<(unsigned)((3 * count + 255) / 256), 256, 0, s->stream>>>(s->n, first, count, s->pos, s->rest);
    return cudaGetLastError();
}
cudaError_t launch_rest_positions(vx_scene* s) { return launch_rest_range(s, 0, s->n); }

cudaError_t launch_velocity(vx_scene* s, double h) {
    if (s->n == 0) return cudaSuccess;
    k_velocity<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->pos, s->vel, s->prev, s->drift, s->pred, s->kin,
                                                          s->tmask, h, s->tile_on);
    return cudaGetLastError();
}

cudaError_t launch_velocity_update(vx_scene* s, uint32_t count, const uint32_t* d_index, const double* d_value,
                                   int32_t op) {
    if (count == 0) return cudaSuccess;
    k_velocity_update<<<(count + 255) / 256, 256, 0, s->stream>>>(s->n, count, d_index, d_value, op, s->vel,
                                                                   s->tmask);
    return cudaGetLastError();
}

}  // namespace vx

using namespace vx;

extern "C" int32_t vx_scene_step(vx_scene* s, const vx_step_params* p, vx_step_stats* out) {
    clear_error();
    if (!s || !p) {
        set_error("vx_scene_step: null argument");
        return VX_BAD_INPUT;
    }
    if (!(p->fixed_dt > 0.0) || !std::isfinite(p->fixed_dt) || p->substeps == 0 || p->corotation_iterations == 0 ||
        !std::isfinite(p->gravity[0]) || !std::isfinite(p->gravity[1]) || !std::isfinite(p->gravity[2])) {
        set_error("vx_scene_step: invalid fixed_dt=%g, substeps=%u, corotation_iterations=%u or gravity",
                  p->fixed_dt, p->substeps, p->corotation_iterations);
        return VX_BAD_INPUT;
    }
    if (p->contact && (!(p->restitution >= 0.0 && p->restitution <= 1.0) || !(p->friction >= 0.0) ||
                       !std::isfinite(p->friction))) {
        set_error("vx_scene_step: invalid restitution=%g or friction=%g", p->restitution, p->friction);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    const double h = p->fixed_dt / (double)p->substeps;
    vx_step_stats st{};
    st.converged = 1;
    int32_t worst = VX_OK;
    for (uint32_t sub = 0; sub < p->substeps; ++sub) {
        cudaError_t e = launch_predict(s, p->gravity, h);
        if (e != cudaSuccess) {
            set_error("vx_scene_step: prediction launch failed: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
        double angle = 0.0;
        int32_t r = vx_fit_rotations(s, &angle);
        if (r != VX_OK) return r;
        st.max_angle = angle;
        for (uint32_t pass = 0; pass < p->corotation_iterations; ++pass) {
            vx_pass_params pp = p->pass;
            pp.h = h;
            pp.reuse_preconditioner = p->pass.reuse_preconditioner && pass > 0;
            vx_pass_stats ps{};
            r = vx_corotational_pass(s, &pp, &ps);
            st.passes += 1;
            st.pcg_iterations += ps.iterations;
            st.residual = ps.residual;
            if (r == VX_NOT_CONVERGED || r == VX_NONFINITE) {
                st.converged = 0;
                if (r == VX_NONFINITE || worst == VX_OK) worst = r;
            } else if (r != VX_OK) {
                return r;
            }
            if (pass + 1 == p->corotation_iterations) break;
            r = vx_fit_rotations(s, &angle);
            if (r != VX_OK) return r;
            st.max_angle = angle;
            if (angle <= p->corotation_tolerance && st.residual <= p->pass.tolerance) break;
        }
        // Velocities come from the solved positions (src/solver.rs:667-681), so
        // they are formed before the contact projection moves positions; the
        // fracture stage then reads the projected ones (src/solver.rs:575-665).
        e = launch_velocity(s, h);
        if (e != cudaSuccess) {
            set_error("vx_scene_step: velocity update failed: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
        if (p->contact) {
            vx_contact_stats cs{};
            r = contact_project(s, &cs, nullptr);
            if (r != VX_OK) return r;
            st.contacts += cs.contacts;
        }
        if (p->fracture) {
            vx_dissipation d{};
            uint32_t broken = 0;
            r = fracture_stage(s, h, &p->fracture_config, &d, &broken);
            if (r != VX_OK) return r;
            st.broken += broken;
            st.dissipation.plastic_heat += d.plastic_heat;
            st.dissipation.stored_plastic += d.stored_plastic;
            st.dissipation.surface_work += d.surface_work;
            st.dissipation.damage_heat += d.damage_heat;
            st.dissipation.released += d.released;
        }
        if (p->contact) {
            vx_contact_heat heat{};
            r = contact_resolve(s, s->drift, p->restitution, p->friction, &heat);
            if (r != VX_OK) return r;
            st.restitution_heat += heat.restitution;
            st.friction_heat += heat.friction;
        }
        e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) {
            set_error("vx_scene_step: velocity update failed: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
    }
    if (out) *out = st;
    if (worst == VX_NONFINITE) set_error("vx_scene_step: non-finite value in a pass");
    else if (worst == VX_NOT_CONVERGED) set_error("vx_scene_step: a pass did not reach its tolerance");
    return worst;
}
