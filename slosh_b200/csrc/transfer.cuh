// Particle/grid transfer kernels of one substep:
//   k_p2g          APIC/MLS particle-to-grid scatter
//   k_grid_update  momentum -> velocity, gravity, clamping, collider BCs
//   k_g2p_update   grid-to-particle gather fused with the particle update
//   k_rigid        rigid-body pose integration
#pragma once

#include "models.cuh"
#include "scene.cuh"

namespace slosh {

// Coordinates of tile node t (tile edge TW) and the rank + local node id of
// the grid block that owns it (the block itself or one of its +1
// neighbours, in slosh's associated-block order).
template <int D>
__device__ __forceinline__ bool tile_node_owner(const DevScene &s, uint32_t r, int t, uint32_t &rank, uint32_t &local) {
    constexpr int TW = Geo<D>::TW, BW = Geo<D>::BW, NN = Geo<D>::NASSOC - 1;
    int c[D];
    c[0] = t % TW;
    if constexpr (D == 3) {
        c[1] = (t / TW) % TW;
        c[2] = t / (TW * TW);
    } else {
        c[1] = t / TW;
    }
    int oct = 0;
    uint32_t loc = 0, mul = 1;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int o = c[k] >= BW ? 1 : 0;
        oct = oct * 2 + o;
        loc += (uint32_t)(c[k] - o * BW) * mul;
        mul *= BW;
    }
    rank = (oct == 0) ? r : s.bnbh[r * NN + oct - 1];
    local = loc;
    return rank != NONE;
}

// Particle-to-grid.  One CTA per active block with primaries; each thread
// scatters whole particles into a shared (block + 2)^D tile of node
// momentum/mass (shared-memory atomics), then the tile is added to the global
// nodes of the block and its +1 neighbours with 16-byte vector atomics.
// Node momentum/mass match slosh's p2g_scatter_style
// (shaders/slosh/solver/p2g_scatter_style.slang:84-154):
//   acc_i = sum_p w_ip [ C_p (x_i - x_p) + m_p v_p + f_p dt ,  m_p ].
template <int D, int NT> __global__ void __launch_bounds__(NT) k_p2g(DevScene s) {
    constexpr int TW = Geo<D>::TW, TILE = Geo<D>::TILE, BW = Geo<D>::BW;
    __shared__ float tile[4][TILE];
    const uint32_t nb = s.ctr->n_blocks;
    const float h = s.h;
    for (uint32_t r = blockIdx.x; r < nb; r += gridDim.x) {
        const uint32_t np = s.bnp[r];
        if (np == 0) continue;
        for (int t = threadIdx.x; t < 4 * TILE; t += NT) (&tile[0][0])[t] = 0.f;
        __syncthreads();
        int bv[D];
        unpack_key<D>(s.bkey[r], bv);
        const uint32_t first = s.bfirst[r];
        for (uint32_t e = threadIdx.x; e < np; e += NT) {
            const uint32_t i = s.perm[first + e];
            const float4 p = s.pm[i];
            const float x[3] = {p.x, p.y, p.z};
            const float m = p.w;
            float d0[D], w[D][3];
            int a[D];
            bool in_block = true;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                const float assoc = rintf(__fdiv_rn(x[k], h)) - 1.0f;
                a[k] = (int)assoc - bv[k] * BW;
                in_block = in_block && a[k] >= 0 && a[k] < BW;
                d0[k] = assoc * h - x[k];
                bspline_weights(__fdiv_rn(-d0[k], h), w[k]);
            }
            if (!in_block) {  // packed-key aliasing far outside the key range
                atomicOr(s.err, ERR_KEY_RANGE);
                continue;
            }
            float q[D], Cm[D][D];
#pragma unroll
            for (int j = 0; j < D; ++j) {
                q[j] = s.vel[j * s.n + i] * m;
                if (s.force_pending) q[j] += s.fdt[j * s.n + i];
#pragma unroll
                for (int k = 0; k < D; ++k) Cm[j][k] = s.C[(j * D + k) * s.n + i];
            }
            float base[D], hc[D][D];  // hc[k] = h * column k of C
#pragma unroll
            for (int j = 0; j < D; ++j) {
                float acc = q[j];
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    acc += Cm[j][k] * d0[k];
                    hc[k][j] = h * Cm[j][k];
                }
                base[j] = acc;
            }
            if constexpr (D == 3) {
#pragma unroll
                for (int sz = 0; sz < 3; ++sz) {
                    float mz[3];
#pragma unroll
                    for (int j = 0; j < 3; ++j) mz[j] = base[j] + (float)sz * hc[2][j];
#pragma unroll
                    for (int sy = 0; sy < 3; ++sy) {
                        float my[3];
#pragma unroll
                        for (int j = 0; j < 3; ++j) my[j] = mz[j] + (float)sy * hc[1][j];
                        const float wyz = w[1][sy] * w[2][sz];
#pragma unroll
                        for (int sx = 0; sx < 3; ++sx) {
                            const float wt = w[0][sx] * wyz;
                            const int idx = (a[0] + sx) + TW * ((a[1] + sy) + TW * (a[2] + sz));
                            atomicAdd(&tile[0][idx], wt * (my[0] + (float)sx * hc[0][0]));
                            atomicAdd(&tile[1][idx], wt * (my[1] + (float)sx * hc[0][1]));
                            atomicAdd(&tile[2][idx], wt * (my[2] + (float)sx * hc[0][2]));
                            atomicAdd(&tile[3][idx], wt * m);
                        }
                    }
                }
            } else {
#pragma unroll
                for (int sy = 0; sy < 3; ++sy) {
                    float my[2];
#pragma unroll
                    for (int j = 0; j < 2; ++j) my[j] = base[j] + (float)sy * hc[1][j];
#pragma unroll
                    for (int sx = 0; sx < 3; ++sx) {
                        const float wt = w[0][sx] * w[1][sy];
                        const int idx = (a[0] + sx) + TW * (a[1] + sy);
                        atomicAdd(&tile[0][idx], wt * (my[0] + (float)sx * hc[0][0]));
                        atomicAdd(&tile[1][idx], wt * (my[1] + (float)sx * hc[0][1]));
                        atomicAdd(&tile[3][idx], wt * m);
                    }
                }
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < TILE; t += NT) {
            const float4 val = make_float4(tile[0][t], tile[1][t], tile[2][t], tile[3][t]);
            if (val.x == 0.f && val.y == 0.f && val.z == 0.f && val.w == 0.f) continue;
            uint32_t rank, local;
            if (!tile_node_owner<D>(s, r, t, rank, local)) continue;
            atomicAdd(&s.nodes[(size_t)rank * 64u + local], val);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Colliders: Sim3/Sim2 poses, ball and cuboid projections, collide() and the
// boundary-condition projection.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void quat_rotate(const float *q, const float *v, float *out) {
    const float t0 = 2.f * (q[1] * v[2] - q[2] * v[1]);
    const float t1 = 2.f * (q[2] * v[0] - q[0] * v[2]);
    const float t2 = 2.f * (q[0] * v[1] - q[1] * v[0]);
    out[0] = v[0] + q[3] * t0 + (q[1] * t2 - q[2] * t1);
    out[1] = v[1] + q[3] * t1 + (q[2] * t0 - q[0] * t2);
    out[2] = v[2] + q[3] * t2 + (q[0] * t1 - q[1] * t0);
}

template <int D> __device__ __forceinline__ void pose_mul_pt(const DevBody &b, const float *p, float *out) {
    if constexpr (D == 3) {
        const float sp[3] = {p[0] * b.scale, p[1] * b.scale, p[2] * b.scale};
        float r[3];
        quat_rotate(b.rot, sp, r);
        for (int i = 0; i < 3; ++i) out[i] = r[i] + b.tra[i];
    } else {
        const float sp0 = p[0] * b.scale, sp1 = p[1] * b.scale;
        out[0] = b.rot[0] * sp0 - b.rot[1] * sp1 + b.tra[0];
        out[1] = b.rot[1] * sp0 + b.rot[0] * sp1 + b.tra[1];
    }
}

template <int D> __device__ __forceinline__ void pose_inv_mul_pt(const DevBody &b, const float *p, float *out) {
    if constexpr (D == 3) {
        const float d[3] = {p[0] - b.tra[0], p[1] - b.tra[1], p[2] - b.tra[2]};
        const float qi[4] = {-b.rot[0], -b.rot[1], -b.rot[2], b.rot[3]};
        float r[3];
        quat_rotate(qi, d, r);
        for (int i = 0; i < 3; ++i) out[i] = r[i] / b.scale;
    } else {
        const float d0 = p[0] - b.tra[0], d1 = p[1] - b.tra[1];
        out[0] = (b.rot[0] * d0 + b.rot[1] * d1) / b.scale;
        out[1] = (-b.rot[1] * d0 + b.rot[0] * d1) / b.scale;
    }
}

// Shape::project_point_on_boundary for balls and cuboids
// (shaders/slosh/rbd/shapes/ball.slang:39-52, cuboid.slang:14-63).
template <int D>
__device__ __forceinline__ bool project_on_boundary(const DevBody &b, const float *pt, float *proj, bool &inside) {
    float local[D], lp[D];
    pose_inv_mul_pt<D>(b, pt, local);
    if (b.shape_type == SLOSH_SHAPE_CUBOID) {
        float outp[D], sgn[D], diff[D], inp[D];
        bool in = true;
#pragma unroll
        for (int i = 0; i < D; ++i) {
            const float shift = fmaxf(-b.sa[i] - local[i], 0.f) - fmaxf(local[i] - b.sa[i], 0.f);
            outp[i] = local[i] + shift;
            const float sw = (local[i] > 0.f) ? 1.f : ((local[i] < 0.f) ? -1.f : 0.f);
            sgn[i] = sw + (fabsf(sw) - 1.f);
            diff[i] = b.sa[i] - sgn[i] * local[i];
            inp[i] = local[i];
            in = in && (local[i] == outp[i]);
        }
        if constexpr (D == 3) {
            const bool px = diff[0] <= diff[1] && diff[0] <= diff[2];
            const bool py = diff[1] <= diff[0] && diff[1] <= diff[2];
            if (px) inp[0] = local[0] + diff[0] * sgn[0];
            else if (py) inp[1] = local[1] + diff[1] * sgn[1];
            else inp[2] = local[2] + diff[2] * sgn[2];
        } else {
            if (diff[0] <= diff[1]) inp[0] = local[0] + diff[0] * sgn[0];
            else inp[1] = local[1] + diff[1] * sgn[1];
        }
#pragma unroll
        for (int i = 0; i < D; ++i) lp[i] = in ? inp[i] : outp[i];
        inside = in;
    } else if (b.shape_type == SLOSH_SHAPE_BALL) {
        float n2 = 0.f;
#pragma unroll
        for (int i = 0; i < D; ++i) n2 += local[i] * local[i];
        const float dist = sqrtf(n2), rad = b.sa[0];
#pragma unroll
        for (int i = 0; i < D; ++i) lp[i] = (dist != 0.f) ? local[i] * (rad / dist) : 0.f;
        if (dist == 0.f) lp[1] = rad;
        inside = dist <= rad;
    } else {
        return false;
    }
    pose_mul_pt<D>(b, lp, proj);
    return true;
}

// collide (shaders/slosh/collision/collide.slang:87-153).  Returns the
// collider id or NONE; `nd` = (normal, dot(point_node - proj, normal)).
template <int D>
__device__ __forceinline__ uint32_t collide(const DevScene &s, const float *pt, float4 &nd) {
    const float cap = s.h * 1.5f;
    float best = 1.0e10f;
    uint32_t id = NONE;
    float bn[D] = {}, bp[D] = {};
    for (uint32_t i = 0; i < s.n_bodies && i < MAX_BODIES; ++i) {
        float proj[D];
        bool inside = false;
        if (!project_on_boundary<D>(s.bodies[i], pt, proj, inside)) continue;
        float dpt[D], n2 = 0.f;
        bool within = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            dpt[k] = proj[k] - pt[k];
            within = within && (fabsf(dpt[k]) <= cap);
            n2 += dpt[k] * dpt[k];
        }
        if (inside || within) {
            const float sign = inside ? -1.f : 1.f;
            const float dist = sqrtf(n2);
            if (sign * dist < best && dist != 0.f) {
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    bn[k] = dpt[k] / (dist * -sign);
                    bp[k] = proj[k];
                }
                id = i;
                best = dist;
            }
        }
    }
    float dd = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) dd += (pt[k] - bp[k]) * bn[k];
    nd = make_float4(bn[0], bn[1], D == 3 ? bn[D - 1] : 0.f, dd);
    return id;
}

// BoundaryCondition::project_velocity (boundary_condition.slang:31-89),
// keeping slosh's use of the collider friction for FrictionZUp.
template <int D>
__device__ __forceinline__ void project_velocity(uint32_t type, float friction, float *vel, const float *n, float dist,
                                                 float dt) {
    if (type == SLOSH_BC_STICK) {
        if (dist <= 0.f)
#pragma unroll
            for (int k = 0; k < D; ++k) vel[k] = 0.f;
    } else if (type == SLOSH_BC_SLIP) {
        if (dist <= 0.f) {
            float nv = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) nv += vel[k] * n[k];
#pragma unroll
            for (int k = 0; k < D; ++k) vel[k] = vel[k] - n[k] * nv;
        }
    } else if (type == SLOSH_BC_SEPARATE || type == SLOSH_BC_FRICTION_Z_UP) {
        float nv = 0.f;
#pragma unroll
        for (int k = 0; k < D; ++k) nv += vel[k] * n[k];
        if (nv < 0.f) {
            if (dist <= 0.f) {
                float tv[D], tl2 = 0.f;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    tv[k] = vel[k] - n[k] * nv;
                    tl2 += tv[k] * tv[k];
                }
                const float tl = sqrtf(tl2);
                const float sc = fmaxf(0.f, tl + friction * nv);
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = ((tl > 1.0e-8f) ? tv[k] / tl : 0.f) * sc;
            } else if (-nv * dt > dist) {
                const float a = dist / dt + nv;
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = vel[k] - a * n[k];
            }
        }
    }
}

// Grid update (shaders/slosh/solver/grid_update.slang:38-163), one thread per
// node.  The collision of a node is reused from the previous substep when
// its block was active there (slosh's cache, which assumes static colliders),
// otherwise collide() runs; both are recorded for the next substep.
template <int D> __global__ void k_grid_update(DevScene s) {
    constexpr int BW = Geo<D>::BW;
    const uint32_t nb = s.ctr->n_blocks;
    const uint32_t stride = gridDim.x * blockDim.x;
    const float h = s.h, dt = s.dt;
    const float vlim = h / dt;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nb * 64u; t += stride) {
        const uint32_t r = t >> 6, node = t & 63u;
        const uint32_t key = s.bkey[r];
        int bv[D], lc[D];
        unpack_key<D>(key, bv);
        if constexpr (D == 3) {
            lc[0] = node & 3;
            lc[1] = (node >> 2) & 3;
            lc[2] = node >> 4;
        } else {
            lc[0] = node & 7;
            lc[1] = node >> 3;
        }
        float cell_pos[D];
#pragma unroll
        for (int k = 0; k < D; ++k) cell_pos[k] = (float)(bv[k] * BW + lc[k]) * h;
        const float4 nv = s.nodes[t];
        const float pm[3] = {nv.x, nv.y, nv.z};
        const float mass = nv.w;
        const float inv_mass = mass > 0.f ? 1.0f / mass : 0.f;
        float vel[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const float v = (pm[k] + mass * s.gravity[k] * dt) * inv_mass;
            vel[k] = fminf(fmaxf(v, -vlim), vlim);
        }
        float4 cn;
        uint32_t cid;
        const uint32_t pslot = hash_find(s.prev_hkeys, s.hcap, key);
        const uint32_t prank = (pslot == NONE) ? NONE : s.prev_hvals[pslot];
        if (prank != NONE) {
            cn = s.prev_coll[(size_t)prank * 64u + node];
            cid = s.prev_coll_id[(size_t)prank * 64u + node];
        } else {
            cid = collide<D>(s, cell_pos, cn);
        }
        s.coll[t] = cn;
        s.coll_id[t] = cid;
        if (cid != NONE) {
            const float n[3] = {cn.x, cn.y, cn.z};
            project_velocity<D>(s.bodies[cid].bc_type, s.bodies[cid].friction, vel, n, cn.w - h, dt);
        }
        s.nodes[t] = make_float4(vel[0], vel[1], D == 3 ? vel[D - 1] : 0.f, mass);
    }
}

// G2P fused with the particle update.  One CTA per active block with
// primaries: the block's (block + 2)^D tile of node velocities is staged in
// shared memory, then each thread gathers v, grad v and div v for its
// particles (g2p.slang:150-265) and applies the particle update of
// particle_update.slang:48-159 with the constitutive model, writing the new
// position, velocity, APIC matrix C and F.
template <int D, int NT> __global__ void __launch_bounds__(NT) k_g2p_update(DevScene s) {
    constexpr int TW = Geo<D>::TW, TILE = Geo<D>::TILE, BW = Geo<D>::BW;
    __shared__ float tv[D][TILE];
    const uint32_t nb = s.ctr->n_blocks;
    const float h = s.h, dt = s.dt;
    const float inv_d = 4.0f / (h * h);
    const float vmax = h / dt;
    const size_t n = s.n;
    for (uint32_t r = blockIdx.x; r < nb; r += gridDim.x) {
        const uint32_t np = s.bnp[r];
        if (np == 0) continue;
        for (int t = threadIdx.x; t < TILE; t += NT) {
            uint32_t rank, local;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (tile_node_owner<D>(s, r, t, rank, local)) v = s.nodes[(size_t)rank * 64u + local];
            tv[0][t] = v.x;
            tv[1][t] = v.y;
            if constexpr (D == 3) tv[2][t] = v.z;
        }
        __syncthreads();
        int bv[D];
        unpack_key<D>(s.bkey[r], bv);
        const uint32_t first = s.bfirst[r];
        for (uint32_t e = threadIdx.x; e < np; e += NT) {
            const uint32_t i = s.perm[first + e];
            const float4 p = s.pm[i];
            const float x[3] = {p.x, p.y, p.z};
            float m = p.w;
            uint32_t fl = s.flags[i];
            // ---- G2P ----
            float vel[D], grad[D][D], div = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                vel[k] = 0.f;
#pragma unroll
                for (int l = 0; l < D; ++l) grad[k][l] = 0.f;
            }
            if (fl & FLAG_ENABLED) {
                float d0[D], w[D][3];
                int a[D];
                bool in_block = true;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const float assoc = rintf(__fdiv_rn(x[k], h)) - 1.0f;
                    a[k] = (int)assoc - bv[k] * BW;
                    in_block = in_block && a[k] >= 0 && a[k] < BW;
                    d0[k] = assoc * h - x[k];
                    bspline_weights(__fdiv_rn(-d0[k], h), w[k]);
                }
                if (!in_block) {  // packed-key aliasing: gather nothing
                    atomicOr(s.err, ERR_KEY_RANGE);
#pragma unroll
                    for (int k = 0; k < D; ++k) a[k] = 0, w[k][0] = w[k][1] = w[k][2] = 0.f;
                }
                if constexpr (D == 3) {
#pragma unroll
                    for (int sz = 0; sz < 3; ++sz)
#pragma unroll
                        for (int sy = 0; sy < 3; ++sy)
#pragma unroll
                            for (int sx = 0; sx < 3; ++sx) {
                                const int idx = (a[0] + sx) + TW * ((a[1] + sy) + TW * (a[2] + sz));
                                const float wt = w[0][sx] * w[1][sy] * w[2][sz];
                                const float nvx = tv[0][idx], nvy = tv[1][idx], nvz = tv[2][idx];
                                const float dp[3] = {d0[0] + (float)sx * h, d0[1] + (float)sy * h,
                                                     d0[2] + (float)sz * h};
                                vel[0] += nvx * wt;
                                vel[1] += nvy * wt;
                                vel[2] += nvz * wt;
                                const float wi = wt * inv_d;
                                const float nvv[3] = {nvx, nvy, nvz};
#pragma unroll
                                for (int c = 0; c < 3; ++c)
#pragma unroll
                                    for (int rr = 0; rr < 3; ++rr) grad[c][rr] += wi * (nvv[c] * dp[rr]);
                                div += wi * (nvx * dp[0] + nvy * dp[1] + nvz * dp[2]);
                            }
                } else {
#pragma unroll
                    for (int sy = 0; sy < 3; ++sy)
#pragma unroll
                        for (int sx = 0; sx < 3; ++sx) {
                            const int idx = (a[0] + sx) + TW * (a[1] + sy);
                            const float wt = w[0][sx] * w[1][sy];
                            const float nvx = tv[0][idx], nvy = tv[1][idx];
                            const float dp[2] = {d0[0] + (float)sx * h, d0[1] + (float)sy * h};
                            vel[0] += nvx * wt;
                            vel[1] += nvy * wt;
                            const float wi = wt * inv_d;
                            const float nvv[2] = {nvx, nvy};
#pragma unroll
                            for (int c = 0; c < 2; ++c)
#pragma unroll
                                for (int rr = 0; rr < 2; ++rr) grad[c][rr] += wi * (nvv[c] * dp[rr]);
                            div += wi * (nvx * dp[0] + nvy * dp[1]);
                        }
                }
            }
            // ---- particle update ----
            const Material &mat = s.materials[fl & FLAG_MAT_MASK];
            const bool fluid = mat.tag == SLOSH_MODEL_FLUID_TAIT;
            const bool sand = mat.tag == SLOSH_MODEL_SAND_LINEAR || mat.tag == SLOSH_MODEL_SAND_NEO_HOOKEAN;
            float len2 = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) len2 += vel[k] * vel[k];
            const float len = sqrtf(len2);
            if (len > vmax)
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = vel[k] / len * h / dt;
            if (s.has_damping) {
                const float dmp = 1.0f + s.damping[i] * dt;
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = vel[k] / dmp;
            }
            const bool fixed = (fl & FLAG_FIXED) != 0;
            if (fixed)
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = 0.f;
            float nx[D];
#pragma unroll
            for (int k = 0; k < D; ++k) nx[k] = x[k] + vel[k] * dt;
            float F[D][D];
#pragma unroll
            for (int rr = 0; rr < D; ++rr)
#pragma unroll
                for (int c = 0; c < D; ++c) F[rr][c] = s.F[(rr * D + c) * n + i];
            if (!fluid) {
                float Fn[D][D];
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        float acc = 0.f;
#pragma unroll
                        for (int k = 0; k < D; ++k) acc += F[k][c] * (grad[rr][k] * dt);
                        Fn[rr][c] = F[rr][c] + acc;
                    }
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) F[rr][c] = Fn[rr][c];
            } else {
                const float f0 = F[0][0];
                const float nf = f0 + f0 * div * dt;
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) F[rr][c] = (rr == c) ? nf : 0.f;
            }
            if (fixed)
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) grad[rr][c] = 0.f;
            float st[3] = {0.f, 0.f, 0.f};
            if (sand)
#pragma unroll
                for (int k = 0; k < 3; ++k) st[k] = s.plastic[k * n + i];
            float tau[D][D];
            model_update<D>(mat, F, st, tau, &s.ctr->n_svd_fp64);
            const float coef = s.V0[i] * inv_d * dt;
            bool finite = true;
#pragma unroll
            for (int k = 0; k < D; ++k) finite = finite && (nx[k] == nx[k]);
            if (finite && det<D>(F) > 0.f) {
                float4 np4 = p;
                np4.x = nx[0];
                np4.y = nx[1];
                if constexpr (D == 3) np4.z = nx[2];
                s.pm[i] = np4;
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) s.C[(rr * D + c) * n + i] = grad[rr][c] * m - tau[rr][c] * coef;
#pragma unroll
                for (int k = 0; k < D; ++k) s.vel[k * n + i] = vel[k];
            } else {
                fl &= ~FLAG_ENABLED;
                s.flags[i] = fl;
                m = 0.f;
                float4 np4 = p;
                np4.w = 0.f;
                s.pm[i] = np4;
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        F[rr][c] = (rr == c) ? 1.f : 0.f;
                        s.C[(rr * D + c) * n + i] = 0.f;
                    }
#pragma unroll
                for (int k = 0; k < D; ++k) s.vel[k * n + i] = 0.f;
            }
#pragma unroll
            for (int rr = 0; rr < D; ++rr)
#pragma unroll
                for (int c = 0; c < D; ++c) s.F[(rr * D + c) * n + i] = F[rr][c];
            if (sand)
#pragma unroll
                for (int k = 0; k < 3; ++k) s.plastic[k * n + i] = st[k];
        }
        __syncthreads();
    }
}

// Rigid-body update (shaders/slosh/solver/rigid_impulses.slang:72-121) with
// integrate_velocity (shaders/slosh/rbd/dynamics/body.slang:117-130).  The
// incremental impulse slosh applies here is never written by any of its
// kernels, so velocity capping (guarded by a non-zero impulse) never runs.
template <int D> __global__ void k_rigid(DevScene s) {
    const uint32_t id = threadIdx.x;
    if (id >= s.n_bodies) return;
    DevBody b = s.bodies[id];
    const float dt = s.dt;
    float init_com[3] = {0.f, 0.f, 0.f};
    pose_mul_pt<D>(b, b.local_com, init_com);
    if constexpr (D == 3) {
        const float sa[3] = {b.angvel[0] * dt, b.angvel[1] * dt, b.angvel[2] * dt};
        const float ang = sqrtf(sa[0] * sa[0] + sa[1] * sa[1] + sa[2] * sa[2]);
        float dq[4] = {0.f, 0.f, 0.f, 1.f};
        if (ang > 0.f) {
            const float sc = sinf(ang * 0.5f) / ang;
            dq[0] = sa[0] * sc;
            dq[1] = sa[1] * sc;
            dq[2] = sa[2] * sc;
            dq[3] = cosf(ang * 0.5f);
        }
        const float rel[3] = {b.tra[0] - init_com[0], b.tra[1] - init_com[1], b.tra[2] - init_com[2]};
        float rr[3];
        quat_rotate(dq, rel, rr);
        for (int k = 0; k < 3; ++k) b.tra[k] = init_com[k] + rr[k] * b.scale + b.linvel[k] * dt;
        const float *q = b.rot;
        float nq[4];
        nq[0] = dq[3] * q[0] + dq[0] * q[3] + dq[1] * q[2] - dq[2] * q[1];
        nq[1] = dq[3] * q[1] - dq[0] * q[2] + dq[1] * q[3] + dq[2] * q[0];
        nq[2] = dq[3] * q[2] + dq[0] * q[1] - dq[1] * q[0] + dq[2] * q[3];
        nq[3] = dq[3] * q[3] - dq[0] * q[0] - dq[1] * q[1] - dq[2] * q[2];
        const float n2 = nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2] + nq[3] * nq[3];
        const float f = 0.5f * (3.0f - n2);
        for (int k = 0; k < 4; ++k) b.rot[k] = nq[k] * f;
    } else {
        const float a = b.angvel[0] * dt;
        const float c = cosf(a), sn = sinf(a);
        const float rel0 = b.tra[0] - init_com[0], rel1 = b.tra[1] - init_com[1];
        const float r0 = c * rel0 - sn * rel1, r1 = sn * rel0 + c * rel1;
        b.tra[0] = init_com[0] + r0 * b.scale + b.linvel[0] * dt;
        b.tra[1] = init_com[1] + r1 * b.scale + b.linvel[1] * dt;
        const float nc = c * b.rot[0] - sn * b.rot[1], ns = sn * b.rot[0] + c * b.rot[1];
        b.rot[0] = nc;
        b.rot[1] = ns;
    }
    for (int k = 0; k < D; ++k) b.linvel[k] = b.linvel[k] + s.gravity[k] * ((b.inv_mass[k] != 0.f) ? 1.f : 0.f) * dt;
    s.bodies[id] = b;
}

}  // namespace slosh
