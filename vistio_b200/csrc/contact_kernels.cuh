// sm_100a kernels of the IPC contact path: collider barriers (ground plane,
// sphere), the CCD step bound, the line-search update and the
// Augmented-Lagrangian bookkeeping of step_with_ipc
// (crates/vistio-solver/src/pd_solver.rs:549-1157).
#pragma once
#include "pd_kernels.cuh"

namespace vistio {

// barrier_gradient (crates/vistio-contact/src/barrier.rs:35-46): squared
// distances, FP64 inside as in the reference.
__device__ __forceinline__ float barrier_grad_dev(float d, float d_hat) {
  float dc = fminf(fmaxf(d, d_hat * 1e-3f), d_hat);
  if (dc >= d_hat) return 0.f;
  double d64 = dc, dh = d_hat, diff = d64 - dh;
  double ln_ratio = log(d64 / dh);
  return float(-(diff) * (2.0 * ln_ratio + diff / d64));
}
// scaled_barrier_gradient (barrier.rs:78-87)
__device__ __forceinline__ float scaled_barrier_grad_dev(float d, float d_hat, float kappa) {
  float r = kappa * barrier_grad_dev(d, d_hat);
  if (isfinite(r)) return r;
  return signbit(r) ? -1e6f : 1e6f;
}
// The same two functions with the squared distance itself in FP64 (the
// reference's f32 clamp constants kept).
__device__ __forceinline__ double barrier_grad64(double d, double d_hat) {
  double dc = fmin(fmax(d, d_hat * double(1e-3f)), d_hat);
  if (dc >= d_hat) return 0.0;
  double diff = dc - d_hat;
  return -diff * (2.0 * log(dc / d_hat) + diff / dc);
}
__device__ __forceinline__ double scaled_barrier_grad64(double d, double d_hat, double kappa) {
  double r = kappa * barrier_grad64(d, d_hat);
  if (isfinite(r)) return r;
  return signbit(r) ? -1e6 : 1e6;
}

__device__ __forceinline__ void warp_sum_u32(uint32_t& v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
}

// Ground and sphere barriers of CollisionPipeline::detect_ipc_contacts
// (collision_pipeline.rs:207-352, ground_plane.rs:68-109, sphere.rs:102-175).
// mode 0: the detect at the start of an AL pass (writes grad / in_contact,
//         records ever-in-contact normals, clears multipliers off contact);
// mode 1: the re-detect after the inner loop (writes grad_up / in_contact_up,
//         reduces active count and max violation).
__global__ void __launch_bounds__(256) k_detect(BatchDev B, int mode) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  const StepParams& P = *B.prm;
  InstRed& R = B.red[ch.x];
  if (R.al_done) return;
  const InstDev I = B.inst[ch.x];
  uint32_t active = 0;
  float viol = 0.f;
  if ((int)threadIdx.x < ch.z) {
    uint32_t g = uint32_t(ch.y) + threadIdx.x;
    float4 x = B.pos[g];
    float3 gr, n;
    bool inc = false;
    // The self-contact gradient was accumulated in FP64 by k_self_grad before
    // this kernel; the collider barriers are added to it in FP64 too: near
    // contact the sphere distance |p - c| - r cancels catastrophically and the
    // log barrier magnifies the rounding, so distance, gradient and normal are
    // formed in double and rounded once.
    double gx = 0.0, gy = 0.0, gz = 0.0, nx = 0.0, ny = 0.0, nz = 0.0, vio = 0.0;
    if (P.self_collision) {
      const double4 s = B.gacc[g];
      gx = s.x; gy = s.y; gz = s.z;
      const double gsq = gx * gx + gy * gy + gz * gz;
      if (gsq > double(1e-12f)) { const double gl = sqrt(gsq); nx = gx / gl; ny = gy / gl; nz = gz / gl; inc = true; }
    }
    const double dh = P.d_hat, kap = P.kappa > 0.f ? P.kappa : I.kappa;
    if (P.has_ground) {
      const double ds = double(x.y) - double(P.ground_h);
      if (ds <= 0.0) {
        vio = fmax(vio, -ds);
        const double dc = fmax(-ds, double(1e-6f));
        active++;
        gy += scaled_barrier_grad64(dc * dc, dh, kap) * 2.0 * dc;
      } else if (ds * ds < dh) {
        active++;
        gy += scaled_barrier_grad64(ds * ds, dh, kap) * 2.0 * ds;
      }
      if (ds * ds < dh || ds <= 0.0) { ny += 1.0; inc = true; }
    }
    if (P.has_sphere) {
      const double dx = double(x.x) - double(P.sphere_c[0]), dy = double(x.y) - double(P.sphere_c[1]),
                   dz = double(x.z) - double(P.sphere_c[2]);
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      const double ds = r - double(P.sphere_r);
      if (ds <= 0.0) {
        vio = fmax(vio, -ds);
        const double dc = fmax(-ds, double(1e-6f));
        active++;
        const double bg = scaled_barrier_grad64(dc * dc, dh, kap);
        if (r > double(1e-6f)) {
          const double f = bg * 2.0 * dc;
          gx += f * (dx / r); gy += f * (dy / r); gz += f * (dz / r);
        } else {
          gy += bg * 2.0 * dc;
        }
      } else if (ds * ds < dh) {
        active++;
        const double f = scaled_barrier_grad64(ds * ds, dh, kap) * 2.0 * ds;
        gx += f * (dx / r); gy += f * (dy / r); gz += f * (dz / r);
      }
      if (ds * ds < dh || ds <= 0.0) {
        if (r > double(1e-6f)) { nx += dx / r; ny += dy / r; nz += dz / r; }
        inc = true;
      }
    }
    // The cylinder and the box contribute barrier gradients only: the
    // reference's pipeline gives them no contact normal (collision_pipeline.rs
    // :305-318), so they leave in_contact / friction / damping alone.
    if (P.has_cyl) {  // CylinderCollider::detect_ipc_contacts (cylinder.rs:121-198)
      const double dx = double(x.x) - double(P.cyl[0]), dz = double(x.z) - double(P.cyl[1]);
      const double dt = double(x.y) - double(P.cyl[2]);  // above the top face when > 0
      const double r = sqrt(dx * dx + dz * dz), ds = r - double(P.cyl[3]);  // outside the wall when > 0
      const double rmin = double(1e-6f);
      double ex = 0.0, ey = 0.0, ez = 0.0, dsq;
      if (dt <= 0.0 && ds <= 0.0) {  // inside: the shorter way out, a tiny distance
        vio = fmax(vio, -fmax(dt, ds));
        if (dt > ds) ey = 1.0;
        else if (r > rmin) { ex = dx / r; ez = dz / r; }
        dsq = double(1e-12f);
      } else if (dt > 0.0 && ds <= 0.0) {  // over the top face
        ey = 1.0;
        dsq = dt * dt;
      } else if (dt <= 0.0) {  // beside the wall
        if (r > rmin) { ex = dx / r; ez = dz / r; }
        dsq = ds * ds;
      } else {  // above and outside: the rim
        if (r > rmin) {
          const double d = sqrt(ds * ds + dt * dt);
          ex = (ds / d) * (dx / r); ey = dt / d; ez = (ds / d) * (dz / r);
        }
        dsq = ds * ds + dt * dt;
      }
      if (dsq < dh && dsq > 0.0) {
        active++;
        const double f = scaled_barrier_grad64(dsq, dh, kap) * 2.0 * sqrt(dsq);
        gx += f * ex; gy += f * ey; gz += f * ez;
      }
    }
    if (P.has_box) {  // BoxCollider::detect_ipc_contacts (box_collider.rs:107-200)
      const double px[3] = {double(x.x), double(x.y), double(x.z)};
      double d[3], q[3], e[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < 3; ++k) {
        const double c = (double(P.box_lo[k]) + double(P.box_hi[k])) * 0.5;
        const double h = (double(P.box_hi[k]) - double(P.box_lo[k])) * 0.5;
        d[k] = px[k] - c;
        q[k] = fabs(d[k]) - h;  // > 0: outside the slab of axis k
      }
      const double mq = fmax(fmax(q[0], q[1]), q[2]);
      double dsq;
      if (mq <= 0.0) {  // inside: out through the nearest face, a tiny distance
        vio = fmax(vio, -mq);
        const int k = mq == q[0] ? 0 : mq == q[1] ? 1 : 2;
        e[k] = copysign(1.0, d[k]);
        dsq = double(1e-12f);
      } else {
        dsq = 0.0;
        for (int k = 0; k < 3; ++k)
          if (q[k] > 0.0) { dsq += q[k] * q[k]; e[k] = q[k] * copysign(1.0, d[k]); }
        const double dl = sqrt(dsq);
        if (dl > double(1e-6f)) { e[0] /= dl; e[1] /= dl; e[2] /= dl; }
      }
      if (dsq < dh && dsq > 0.0) {
        active++;
        const double f = scaled_barrier_grad64(dsq, dh, kap) * 2.0 * sqrt(dsq);
        gx += f * e[0]; gy += f * e[1]; gz += f * e[2];
      }
    }
    if (inc) {
      const double ls = nx * nx + ny * ny + nz * nz;
      if (ls > double(1e-12f)) { const double il = 1.0 / sqrt(ls); nx *= il; ny *= il; nz *= il; }
    }
    gr = make_float3(float(gx), float(gy), float(gz));
    n = make_float3(float(nx), float(ny), float(nz));
    viol = fmaxf(viol, float(vio));
    float4 g4 = make_float4(gr.x, gr.y, gr.z, 0.f);
    if (mode == 0) {
      B.grad[g] = g4;
      B.in_contact[g] = inc;
      if (inc) { B.ever[g] = 1; B.fin_n[g] = make_float4(n.x, n.y, n.z, 0.f); }
      else B.lam[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      B.grad_up[g] = g4;
      B.in_contact_up[g] = inc;
      if (inc) { B.ever[g] = 1; B.fin_n[g] = make_float4(n.x, n.y, n.z, 0.f); }
    }
  }
  if (mode == 1) {
    warp_sum_u32(active);
    for (int o = 16; o > 0; o >>= 1) viol = fmaxf(viol, __shfl_down_sync(0xffffffffu, viol, o));
    if ((threadIdx.x & 31) == 0) {
      if (active) atomicAdd(&R.active, active);
      if (viol > 0.f) atomicMax(&R.maxviol_bits, __float_as_uint(viol));
    }
  }
  (void)I;
}

// CCD step bound for the colliders (ground_plane.rs:112-134, sphere.rs:178-224,
// cylinder.rs:201-262, box_collider.rs:203-251)
// and the backtracking sum grad . d over free vertices (pd_solver.rs:915-925).
__global__ void __launch_bounds__(256) k_ccd(BatchDev B) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  const StepParams& P = *B.prm;
  InstRed& R = B.red[ch.x];
  if (R.al_done) return;
  const InstDev I = B.inst[ch.x];
  float toi = 1.f;
  double gdd = 0.0;
  if ((int)threadIdx.x < ch.z) {
    uint32_t g = uint32_t(ch.y) + threadIdx.x;
    float4 x0 = B.pos[g];
    float4 d = B.Y[I.vbase + B.perm_local[g]];
    float3 x1 = make_float3(x0.x + d.x, x0.y + d.y, x0.z + d.z);
    if (P.has_ground) {
      float y0 = x0.y, y1 = x1.y, h = P.ground_h;
      if (y0 > h && y1 < h) {
        float t = (h - y0) / (y1 - y0);
        if (t >= 0.f && t <= 1.f) toi = fminf(toi, t * 0.9f);
      }
    }
    if (P.has_sphere) {
      float r2 = P.sphere_r * P.sphere_r;
      float px0 = x0.x - P.sphere_c[0], py0 = x0.y - P.sphere_c[1], pz0 = x0.z - P.sphere_c[2];
      float px1 = x1.x - P.sphere_c[0], py1 = x1.y - P.sphere_c[1], pz1 = x1.z - P.sphere_c[2];
      if (!(px0 * px0 + py0 * py0 + pz0 * pz0 < r2)) {
        float vx = px1 - px0, vy = py1 - py0, vz = pz1 - pz0;
        float a = vx * vx + vy * vy + vz * vz;
        float b = 2.f * (px0 * vx + py0 * vy + pz0 * vz);
        float c = px0 * px0 + py0 * py0 + pz0 * pz0 - r2;
        if (a > 1e-8f) {
          float disc = b * b - 4.f * a * c;
          if (disc >= 0.f) {
            float t = (-b - sqrtf(disc)) / (2.f * a);
            if (t >= 0.f && t <= 1.f) toi = fminf(toi, t * 0.9f);
          }
        }
      }
    }
    if (P.has_cyl) {
      const float r2 = P.cyl[3] * P.cyl[3];
      const float px0 = x0.x - P.cyl[0], py0 = x0.y - P.cyl[2], pz0 = x0.z - P.cyl[1];
      const float vx = (x1.x - P.cyl[0]) - px0, vy = (x1.y - P.cyl[2]) - py0, vz = (x1.z - P.cyl[1]) - pz0;
      // the endless wall: |(p0 + t v)_xz| = r, first root, hit below the top face
      const float a = vx * vx + vz * vz, b = 2.f * (px0 * vx + pz0 * vz), c = px0 * px0 + pz0 * pz0 - r2;
      if (a > 1e-8f) {
        const float disc = b * b - 4.f * a * c;
        if (disc >= 0.f) {
          const float t = (-b - sqrtf(disc)) / (2.f * a);
          if (t >= 0.f && t <= 1.f && py0 + t * vy <= 0.f) toi = fminf(toi, t * 0.9f);
        }
      }
      // the top face: crossing y = top inside the radius
      if (vy < -1e-8f && py0 > 0.f) {
        const float t = -py0 / vy;
        if (t >= 0.f && t <= 1.f) {
          const float xh = px0 + t * vx, zh = pz0 + t * vz;
          if (xh * xh + zh * zh <= r2) toi = fminf(toi, t * 0.9f);
        }
      }
    }
    if (P.has_box) {  // slab test: the entry time into the box during the step
      const float p0[3] = {x0.x, x0.y, x0.z}, v[3] = {x1.x - x0.x, x1.y - x0.y, x1.z - x0.z};
      float tmin = 0.f, tmax = 1.f;
      bool hit = true;
      for (int k = 0; k < 3 && hit; ++k) {
        if (fabsf(v[k]) < 1e-8f) {
          hit = p0[k] >= P.box_lo[k] && p0[k] <= P.box_hi[k];
        } else {
          float t1 = (P.box_lo[k] - p0[k]) / v[k], t2 = (P.box_hi[k] - p0[k]) / v[k];
          if (t1 > t2) { const float tt = t1; t1 = t2; t2 = tt; }
          tmin = fmaxf(tmin, t1);
          tmax = fminf(tmax, t2);
          hit = tmin <= tmax && tmax >= 0.f;
        }
      }
      if (hit && tmin >= 0.f && tmin <= 1.f) toi = fminf(toi, tmin * 0.9f);
    }
    if (!B.pinned[g]) {
      float4 gr = B.grad[g];
      gdd = double(gr.x * d.x + gr.y * d.y + gr.z * d.z);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    toi = fminf(toi, __shfl_down_sync(0xffffffffu, toi, o));
    gdd += __shfl_down_sync(0xffffffffu, gdd, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (toi < 1.f) atomicMin(&R.toi_bits, __float_as_uint(fmaxf(toi, 0.f)));
    if (gdd != 0.0) atomicAdd(&R.gdd, gdd);
  }
}

// The colliders of the runner's non-IPC path (runner.rs:212-218 then
// CollisionPipeline::step, collision_pipeline.rs:117-199, with no mesh or self
// contact): after a plain step, GroundPlane, GroundPlane again, SphereCollider,
// CylinderCollider and BoxCollider ::resolve, in that order, on every free
// vertex (ground_plane.rs:26-65, sphere.rs:29-100, cylinder.rs:30-118,
// box_collider.rs:26-99): a vertex inside is moved to the surface, its
// velocity loses the inward part and is damped. FP32 like the reference.
struct ColliderDev {
  int32_t has_ground, has_sphere, has_cyl, has_box;
  float ground_h, sc[3], sr, cyl[4], lo[3], hi[3];
};

// Separately rounded FP32 operations: the projections below are written
// without fused multiply-adds, so each vertex lands on the same float the
// reference's scalar Rust code computes.
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rdot3(float a, float b, float c, float x, float y, float z) {
  return radd(radd(rmul(a, x), rmul(b, y)), rmul(c, z));
}

__device__ __forceinline__ void resolve_ground(const ColliderDev& C, float4& x, float4& v, float4& pv, uint32_t& n,
                                               float& pen, float& f) {
  const float depth = rsub(C.ground_h, x.y);
  if (depth > 0.f) {
    x.y = C.ground_h;
    pv.y = C.ground_h;  // the velocity (x - prev) / dt is not to point down
    v.x = rmul(v.x, 0.5f); v.z = rmul(v.z, 0.5f);
    if (v.y < 0.f) v.y = 0.f;
    ++n;
    pen = fmaxf(pen, depth);
    f = radd(f, depth);
  }
}

// Per instance i and collider c (ground, sphere, cylinder, box), the
// ContactResult fields of CollisionStepResult: out[8i+2c] += vertices
// resolved, out[8i+2c+1] = max(itself, the float bits of the deepest
// penetration) and force[4i+c] += the sum of the depths. The second ground
// pass finds nothing the first left and is not counted, as in the reference.
__global__ void __launch_bounds__(256) k_resolve(BatchDev B, ColliderDev C, uint32_t* out, double* force) {
  int4 ch = B.vtx_chunks[blockIdx.x];
  uint32_t n[4] = {0, 0, 0, 0};
  float pen[4] = {0.f, 0.f, 0.f, 0.f}, f[4] = {0.f, 0.f, 0.f, 0.f};
  if ((int)threadIdx.x < ch.z) {
    const uint32_t g = uint32_t(ch.y) + threadIdx.x;
    if (!B.pinned[g] && B.mass[g] > 1e-12f) {  // inv_mass != 0 (state.rs:108-116)
      float4 x = B.pos[g], v = B.vel[g], pv = B.prev[g];
      if (C.has_ground) {
        resolve_ground(C, x, v, pv, n[0], pen[0], f[0]);
        uint32_t n2 = 0;
        float p2 = 0.f, f2 = 0.f;
        resolve_ground(C, x, v, pv, n2, p2, f2);
      }
      if (C.has_sphere) {
        const float r = C.sr, r2 = rmul(r, r);
        const float dx = rsub(x.x, C.sc[0]), dy = rsub(x.y, C.sc[1]), dz = rsub(x.z, C.sc[2]);
        const float d2 = rdot3(dx, dy, dz, dx, dy, dz);
        if (d2 < r2 && d2 > 1e-12f) {
          const float d = __fsqrt_rn(d2), depth = rsub(r, d);
          const float nx = __fdiv_rn(dx, d), ny = __fdiv_rn(dy, d), nz = __fdiv_rn(dz, d);
          x.x = radd(x.x, rmul(nx, depth)); x.y = radd(x.y, rmul(ny, depth)); x.z = radd(x.z, rmul(nz, depth));
          const float vn = rdot3(v.x, v.y, v.z, nx, ny, nz);
          if (vn < 0.f) {  // the normal part goes, the tangential part keeps half (friction 0.5)
            v.x = rmul(rsub(v.x, rmul(nx, vn)), 0.5f);
            v.y = rmul(rsub(v.y, rmul(ny, vn)), 0.5f);
            v.z = rmul(rsub(v.z, rmul(nz, vn)), 0.5f);
          }
          ++n[1];
          pen[1] = fmaxf(pen[1], depth);
          f[1] = radd(f[1], depth);
        } else if (d2 <= 1e-12f) {  // at the centre: straight up, at rest
          x.y = radd(x.y, r);
          v.x = 0.f; v.y = 0.f; v.z = 0.f;
          ++n[1];
          pen[1] = fmaxf(pen[1], r);
          f[1] = radd(f[1], r);
        }
      }
      if (C.has_cyl && !(x.y > C.cyl[2])) {  // only below the top face: the cylinder reaches down without end
        const float r = C.cyl[3];
        const float dx = rsub(x.x, C.cyl[0]), dz = rsub(x.z, C.cyl[1]);
        const float d2 = radd(rmul(dx, dx), rmul(dz, dz));
        if (d2 < rmul(r, r)) {
          const float d = __fsqrt_rn(d2), side = rsub(r, d), top = rsub(C.cyl[2], x.y);
          bool up = top < side;
          if (pv.y >= C.cyl[2]) up = true;  // it was above the top a frame ago: it came through the top
          if (d < 1e-12f) up = true;
          if (up) {
            x.y = C.cyl[2];
            if (v.y < 0.f) v.y = 0.f;
            v.x = rmul(v.x, 0.1f); v.z = rmul(v.z, 0.1f);
            pen[2] = fmaxf(pen[2], top);
            f[2] = radd(f[2], top);
          } else {
            if (d > 1e-12f) {
              const float nx = __fdiv_rn(dx, d), nz = __fdiv_rn(dz, d);
              x.x = radd(x.x, rmul(nx, side)); x.z = radd(x.z, rmul(nz, side));
              const float vn = radd(rmul(v.x, nx), rmul(v.z, nz));
              if (vn < 0.f) { v.x = rsub(v.x, rmul(vn, nx)); v.z = rsub(v.z, rmul(vn, nz)); }
              v.y = rmul(v.y, 0.7f);
            }
            pen[2] = fmaxf(pen[2], side);
            f[2] = radd(f[2], side);
          }
          ++n[2];
        }
      }
      if (C.has_box && x.x >= C.lo[0] && x.x <= C.hi[0] && x.y >= C.lo[1] && x.y <= C.hi[1] && x.z >= C.lo[2] &&
          x.z <= C.hi[2]) {
        const float dnx = rsub(x.x, C.lo[0]), dpx = rsub(C.hi[0], x.x), dny = rsub(x.y, C.lo[1]);
        const float dpy = rsub(C.hi[1], x.y), dnz = rsub(x.z, C.lo[2]), dpz = rsub(C.hi[2], x.z);
        float md = fminf(fminf(fminf(fminf(fminf(dnx, dpx), dny), dpy), dnz), dpz);
        if (pv.y >= C.hi[1]) md = dpy;  // it came through the top
        const float fr = 0.7f;  // faces tried in the order -x, +x, +y, -y, +z, -z
        if (md == dnx) { x.x = C.lo[0]; if (v.x > 0.f) v.x = 0.f; v.y = rmul(v.y, fr); v.z = rmul(v.z, fr); }
        else if (md == dpx) { x.x = C.hi[0]; if (v.x < 0.f) v.x = 0.f; v.y = rmul(v.y, fr); v.z = rmul(v.z, fr); }
        else if (md == dpy) { x.y = C.hi[1]; if (v.y < 0.f) v.y = 0.f; v.x = rmul(v.x, fr); v.z = rmul(v.z, fr); }
        else if (md == dny) { x.y = C.lo[1]; if (v.y > 0.f) v.y = 0.f; v.x = rmul(v.x, fr); v.z = rmul(v.z, fr); }
        else if (md == dpz) { x.z = C.hi[2]; if (v.z < 0.f) v.z = 0.f; v.x = rmul(v.x, fr); v.y = rmul(v.y, fr); }
        else if (md == dnz) { x.z = C.lo[2]; if (v.z > 0.f) v.z = 0.f; v.x = rmul(v.x, fr); v.y = rmul(v.y, fr); }
        ++n[3];
        pen[3] = fmaxf(pen[3], md);
        f[3] = radd(f[3], md);
      }
      B.pos[g] = x; B.vel[g] = v; B.prev[g] = pv;
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint32_t k = n[c];
    float p = pen[c];
    double t = f[c];
    warp_sum_u32(k);
    for (int o = 16; o > 0; o >>= 1) {
      p = fmaxf(p, __shfl_down_sync(0xffffffffu, p, o));
      t += __shfl_down_sync(0xffffffffu, t, o);
    }
    if ((threadIdx.x & 31) == 0 && k) {
      atomicAdd(out + 8 * ch.x + 2 * c, k);
      atomicMax(out + 8 * ch.x + 2 * c + 1, __float_as_uint(p));  // non-negative floats order like their bits
      atomicAdd(force + 4 * ch.x + c, t);
    }
  }
}

// Step-size selection (pd_solver.rs:896-932) and x <- x + alpha d on free vertices.
__global__ void __launch_bounds__(256) k_ipc_update(BatchDev B) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  InstRed& R = B.red[ch.x];
  if (R.al_done) return;
  const InstDev I = B.inst[ch.x];
  float max_alpha = fmaxf(__uint_as_float(R.toi_bits), 1e-6f);
  if (max_alpha < 1.f) max_alpha *= 0.8f;
  max_alpha = fminf(max_alpha, 1.f);
  float alpha = max_alpha;
  for (int bt = 0; bt < 4; ++bt) {
    if (alpha < 0.1f) break;
    if (R.gdd * double(R.mu) > double(1e-4f) * R.diff_sq * 100.0) alpha *= 0.5f;
    else break;
  }
  if (threadIdx.x == 0 && ch.y == int(I.vbase)) R.alpha = alpha;
  if ((int)threadIdx.x >= ch.z) return;
  uint32_t g = uint32_t(ch.y) + threadIdx.x;
  if (B.pinned[g]) return;
  float4 d = B.Y[I.vbase + B.perm_local[g]];
  float4 x = B.pos[g];
  x.x += alpha * d.x; x.y += alpha * d.y; x.z += alpha * d.z;
  B.pos[g] = x;
}

// Clears the re-detect reductions before the inner loop of an AL pass.
__global__ void k_al_begin(BatchDev B, uint32_t ninst) {
  pdl_begin();
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ninst) return;
  InstRed& R = B.red[k];
  if (R.al_done) return;
  R.active = 0;
  R.maxviol_bits = 0;
}

// lambda += mu * grad_up on re-detected contacts when the AL pass did not
// converge (pd_solver.rs:1005-1018).
__global__ void __launch_bounds__(256) k_al_end(BatchDev B) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  const StepParams& P = *B.prm;
  InstRed& R = B.red[ch.x];
  if (R.al_done) return;
  if ((int)threadIdx.x >= ch.z) return;
  if (__uint_as_float(R.maxviol_bits) < P.al_tolerance) return;
  uint32_t g = uint32_t(ch.y) + threadIdx.x;
  if (!B.in_contact_up[g]) return;
  float4 gu = B.grad_up[g], la = B.lam[g];
  float mu = R.mu;
  la.x += mu * gu.x; la.y += mu * gu.y; la.z += mu * gu.z;
  B.lam[g] = la;
}

// Per instance: count the pass, record the active contacts, stop or grow mu.
__global__ void k_al_finish(BatchDev B, uint32_t ninst) {
  pdl_begin();
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ninst) return;
  const StepParams& P = *B.prm;
  InstRed& R = B.red[k];
  if (R.al_done) return;
  R.al_iters += 1;
  R.last_active = R.active;
  if (__uint_as_float(R.maxviol_bits) < P.al_tolerance) R.al_done = 1;
  else R.mu *= P.al_mu_growth;
}

// Zeroes the FP64 self-contact gradient accumulator before a detect.
__global__ void __launch_bounds__(256) k_clear_grad(BatchDev B) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  if (B.red[ch.x].al_done) return;
  if ((int)threadIdx.x >= ch.z) return;
  uint32_t g = uint32_t(ch.y) + threadIdx.x;
  B.gacc[g] = make_double4(0.0, 0.0, 0.0, 0.0);
}

}  // namespace vistio
