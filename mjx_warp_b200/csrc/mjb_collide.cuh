// Collision detection and constraint assembly, one warp per world.
//
// Broadphase: the reference's nxn test (collision_driver.py:458-512) evaluated over the geom pairs
// that survive the model-only filter (_geom_filter, :27-49 — contype/conaffinity, weld and
// parent-child rules), which put_model precomputes in nxn element order.  The bounding test is
// evaluated with explicitly rounded float operations (no FMA contraction), so given the same
// geom poses it decides exactly as a non-contracting FP32 evaluation of the reference predicate.
// Each world reserves one contiguous block of collision_pair / contact / efc rows with a single
// atomic on the global counter, and writes its entries there in canonical order (pair order, then
// contact index; limit rows, then 4 pyramid rows per contact).
#pragma once

#include "mjb_world.cuh"

namespace mjb {

__device__ __forceinline__ float rdot3(float ax, float ay, float az, float bx, float by, float bz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// collision_driver.py:480-503 (bounding sphere / plane half-space test)
__device__ __forceinline__ bool nxn_bound(const MjbModel& m, const float* gxpos, const float* gxmat,
                                          int g1, int g2) {
  const float s1 = m.geom_rbound[g1], s2 = m.geom_rbound[g2];
  const float bound = __fadd_rn(__fadd_rn(s1, s2), fmaxf(m.geom_margin[g1], m.geom_margin[g2]));
  const float dx = __fsub_rn(gxpos[3 * g2], gxpos[3 * g1]);
  const float dy = __fsub_rn(gxpos[3 * g2 + 1], gxpos[3 * g1 + 1]);
  const float dz = __fsub_rn(gxpos[3 * g2 + 2], gxpos[3 * g1 + 2]);
  if (s1 != 0.f && s2 != 0.f) return rdot3(dx, dy, dz, dx, dy, dz) <= __fmul_rn(bound, bound);
  if (s1 == 0.f) {
    const float* x = gxmat + 9 * g1;
    return rdot3(dx, dy, dz, x[2], x[5], x[8]) <= bound;
  }
  const float* x = gxmat + 9 * g2;
  return rdot3(-dx, -dy, -dz, x[2], x[5], x[8]) <= bound;
}

// Reserves `count` entries of a flat array on the global counter; returns the base index, or -1
// (and sets `flag` in the world status) when the block does not fit within `cap`.
__device__ __forceinline__ int reserve(int* counter, int count, int cap, uint32_t* status,
                                       uint32_t flag, int lane) {
  int adr = 0;
  if (lane == 0 && count > 0) {
    adr = atomicAdd(counter, count);
    if (adr + count > cap) {
      if (status) atomicOr(status, flag);
      adr = -1;
    }
  }
  return __shfl_sync(WARP_FULL, adr, 0);
}

// collision_driver.py:458-512 + _add_geom_pair (:52-68)
__device__ void nxn_broadphase(const MjbModel& m, const MjbData& d, int w, int lane) {
  const float* gxpos = d.geom_xpos + W(w, 3 * m.ngeom);
  const float* gxmat = d.geom_xmat + W(w, 9 * m.ngeom);
  const int np = m.npair_cand;
  int count = 0;
  unsigned passed = 0u;  // the lane's test results for the first 32 chunks, kept for the write pass
  for (int base = 0, chunk = 0; base < np; base += 32, chunk++) {
    const int e = base + lane;
    const bool pass = e < np && nxn_bound(m, gxpos, gxmat, m.pair_cand[2 * e], m.pair_cand[2 * e + 1]);
    if (pass && chunk < 32) passed |= 1u << chunk;
    count += __popc(__ballot_sync(WARP_FULL, pass));
  }
  const int adr = reserve(d.ncollision, count, d.nconmax, d.world_status ? d.world_status + w : nullptr,
                          MJB_WS_PAIR_OVERFLOW, lane);
  if (adr < 0) count = 0;
  if (count > 0) {
    int run = 0;
    for (int base = 0, chunk = 0; base < np; base += 32, chunk++) {
      const int e = base + lane;
      int g1 = 0, g2 = 0;
      bool pass = false;
      if (e < np) {
        g1 = m.pair_cand[2 * e];
        g2 = m.pair_cand[2 * e + 1];
        pass = chunk < 32 ? ((passed >> chunk) & 1u) != 0u : nxn_bound(m, gxpos, gxmat, g1, g2);
      }
      const unsigned mask = __ballot_sync(WARP_FULL, pass);
      if (pass) {
        const int k = adr + run + __popc(mask & ((1u << lane) - 1u));
        const bool swap = m.geom_type[g1] > m.geom_type[g2];
        d.collision_pair[2 * k] = swap ? g2 : g1;
        d.collision_pair[2 * k + 1] = swap ? g1 : g2;
        d.collision_worldid[k] = w;
      }
      run += __popc(mask);
    }
  }
  if (lane == 0) {
    d.world_pairadr[w] = adr < 0 ? 0 : adr;
    d.world_npair[w] = count;
  }
  __syncwarp();
}

// ------------------------------------------------------------------------------------------
// Sweep-and-prune broadphase (collision_driver.py:71-301, 350-455), one warp per world.
//
// Each geom's bounding sphere (rbound + margin; planes get radius 1e9) is projected on the fixed
// sweep direction normalize(0.5935, 0.7790, 0.1235); the lower bounds are sorted with their geom
// ids (a bitonic sort of the world's keys in the warp's shared memory, ties in geom-id order as a
// stable radix sort leaves them); sorted position i is then tested against positions
// i+1 .. limit, limit = min(ngeom - 1, first position whose lower bound exceeds i's upper bound)
// (a binary search; the reference's range includes that first position), with the model filter
// (_geom_filter, :27-49) and the reference's overlap test on the sorted spheres and encoded planes
// (:163-184).  Pairs are written in sweep order (position i ascending, then j), with the
// type-ordering swap of _add_geom_pair; the reference appends them with an atomic counter.
//
// encode_plane / decode_plane are restated as the reference evaluates them, including
// decode_plane taking the length of the whole 4-vector (the w code -2 or -3 included) as the
// plane offset's magnitude; for planes through the origin (code -1) the offset is 0.
//
// Shared memory per warp (sap_smem_floats): sorted spheres / planes (float4, ngeom), sorted lower
// bounds and geom ids (padded to a power of two), upper bounds by geom id, per-position counts.

__host__ __device__ __forceinline__ int sap_pow2(int n) {
  int p = 32;
  while (p < n) p <<= 1;
  return p;
}
// a multiple of 4 floats, so every warp's slice (and its float4 array) stays 16-byte aligned
__host__ __device__ __forceinline__ int sap_smem_floats(int ngeom) {
  return (4 * ngeom + 2 * sap_pow2(ngeom) + 2 * ngeom + 3) & ~3;
}

// collision_driver.py:27-49
__device__ __forceinline__ bool geom_filter(const MjbModel& m, int g1, int g2, bool filterparent) {
  const int b1 = m.geom_bodyid[g1], b2 = m.geom_bodyid[g2];
  const int w1 = m.body_weldid[b1], w2 = m.body_weldid[b2];
  const int wp1 = m.body_weldid[m.body_parentid[w1]], wp2 = m.body_weldid[m.body_parentid[w2]];
  const bool self = w1 == w2;
  const bool pc = filterparent && w1 != 0 && w2 != 0 && (w1 == wp2 || w2 == wp1);
  const bool mask = (m.geom_contype[g1] & m.geom_conaffinity[g2]) ||
                    (m.geom_contype[g2] & m.geom_conaffinity[g1]);
  return mask && !self && !pc;
}

// wp.normalize: the vector divided by its length
__device__ __forceinline__ void sap_normalize(float& x, float& y, float& z) {
  const float l = __fsqrt_rn(rdot3(x, y, z, x, y, z));
  if (l > 0.f) {
    x = __fdiv_rn(x, l);
    y = __fdiv_rn(y, l);
    z = __fdiv_rn(z, l);
  }
}

// collision_driver.py:98-118
__device__ __forceinline__ float4 sap_encode_plane(float nx, float ny, float nz, float px, float py,
                                                   float pz, float margin) {
  sap_normalize(nx, ny, nz);
  const float off = -rdot3(nx, ny, nz, __fadd_rn(px, __fmul_rn(nx, margin)),
                           __fadd_rn(py, __fmul_rn(ny, margin)), __fadd_rn(pz, __fmul_rn(nz, margin)));
  const float scale = fabsf(off);
  if (fabsf(off) < 1e-6f) return make_float4(nx, ny, nz, -1.f);
  return make_float4(__fmul_rn(scale, nx), __fmul_rn(scale, ny), __fmul_rn(scale, nz),
                     off < 0.f ? -2.f : -3.f);
}

// collision_driver.py:121-130 (normal, offset)
__device__ __forceinline__ float4 sap_decode_plane(float4 e) {
  const float mag = __fsqrt_rn(__fadd_rn(rdot3(e.x, e.y, e.z, e.x, e.y, e.z), __fmul_rn(e.w, e.w)));
  float nx = e.x, ny = e.y, nz = e.z;
  sap_normalize(nx, ny, nz);
  const float off = e.w == -1.f ? 0.f : (e.w == -2.f ? -mag : mag);
  return make_float4(nx, ny, nz, off);
}

// collision_driver.py:163-184
__device__ __forceinline__ bool sap_overlap(float4 a, float4 b) {
  if (a.w < 0.f && b.w < 0.f) return false;
  if (a.w < 0.f || b.w < 0.f) {
    if (b.w < 0.f) {
      const float4 t = a;
      a = b;
      b = t;
    }
    const float4 p = sap_decode_plane(a);
    const float dist = __fadd_rn(rdot3(b.x, b.y, b.z, p.x, p.y, p.z), p.w);
    return dist <= b.w;
  }
  const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
  const float r = __fadd_rn(a.w, b.w);
  return rdot3(dx, dy, dz, dx, dy, dz) <= __fmul_rn(r, r);
}

__device__ void sap_broadphase(const MjbModel& m, const MjbData& d, int w, int lane, float* sm) {
  const int ng = m.ngeom, P = sap_pow2(ng);
  float4* S = reinterpret_cast<float4*>(sm);
  float* lo = sm + 4 * ng;
  int* idx = reinterpret_cast<int*>(lo + P);
  float* up = lo + 2 * P;
  int* cnt = reinterpret_cast<int*>(up + ng);
  const float* gxpos = d.geom_xpos + W(w, 3 * ng);
  const float* gxmat = d.geom_xmat + W(w, 9 * ng);
  float dx = 0.5935f, dy = 0.7790f, dz = 0.1235f;
  sap_normalize(dx, dy, dz);
  // broadphase_project_spheres_onto_sweep_direction_kernel (:72-92)
  for (int g = lane; g < P; g += 32) {
    if (g < ng) {
      float r = m.geom_rbound[g];
      if (r == 0.f) r = 1e9f;
      const float sr = __fadd_rn(r, m.geom_margin[g]);
      const float c = rdot3(dx, dy, dz, gxpos[3 * g], gxpos[3 * g + 1], gxpos[3 * g + 2]);
      lo[g] = __fsub_rn(c, sr);
      up[g] = __fadd_rn(c, sr);
      idx[g] = g;
    } else {
      lo[g] = __int_as_float(0x7f800000);
      idx[g] = g;
    }
  }
  __syncwarp();
  // sort (lower bound, geom id) ascending
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = lane; t < P / 2; t += 32) {
        const int a = 2 * j * (t / j) + (t % j), b = a + j;
        const float ka = lo[a], kb = lo[b];
        const int ia = idx[a], ib = idx[b];
        const bool gt = ka > kb || (ka == kb && ia > ib);
        if (gt == ((a & k) == 0)) {
          lo[a] = kb;
          lo[b] = ka;
          idx[a] = ib;
          idx[b] = ia;
        }
      }
      __syncwarp();
    }
  }
  // reorder_bounding_spheres_kernel (:134-156)
  for (int i = lane; i < ng; i += 32) {
    const int g = idx[i];
    const float* c = gxpos + 3 * g;
    const float r = m.geom_rbound[g], margin = m.geom_margin[g];
    if (r == 0.f) {
      const float* x = gxmat + 9 * g;
      S[i] = sap_encode_plane(x[2], x[5], x[8], c[0], c[1], c[2], margin);
    } else {
      S[i] = make_float4(c[0], c[1], c[2], __fadd_rn(r, margin));
    }
  }
  __syncwarp();
  const bool filterparent = !(m.disableflags & DSBL_FILTERPARENT);
  // sap_broadphase_prepare_kernel (:219-236) + sap_broadphase_kernel (:272-300), per position i
  auto sweep = [&](int i, int out) {
    const int g1 = idx[i];
    const float end = up[g1];
    int a = i + 1, b = ng;
    while (a < b) {
      const int mid = (a + b) >> 1;
      if (lo[mid] > end) b = mid;
      else a = mid + 1;
    }
    const int limit = min(ng - 1, a);
    int n = 0;
    for (int j = i + 1; j <= limit; j++) {
      const int g2 = idx[j];
      if (!geom_filter(m, g1, g2, filterparent) || !sap_overlap(S[i], S[j])) continue;
      if (out >= 0) {
        const int k = out + n;
        const bool swap = m.geom_type[g1] > m.geom_type[g2];
        d.collision_pair[2 * k] = swap ? g2 : g1;
        d.collision_pair[2 * k + 1] = swap ? g1 : g2;
        d.collision_worldid[k] = w;
      }
      n++;
    }
    return n;
  };
  int total = 0;
  for (int i = lane; i < ng; i += 32) {
    cnt[i] = sweep(i, -1);
    total += cnt[i];
  }
  total = warp_sum_i(total);
  const int adr = reserve(d.ncollision, total, d.nconmax, d.world_status ? d.world_status + w : nullptr,
                          MJB_WS_PAIR_OVERFLOW, lane);
  if (adr < 0) total = 0;
  if (total > 0) {
    int run = adr;
    for (int base = 0; base < ng; base += 32) {
      const int i = base + lane;
      const int c = i < ng ? cnt[i] : 0;
      int incl = c;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(WARP_FULL, incl, o);
        if (lane >= o) incl += v;
      }
      if (c > 0) sweep(i, run + incl - c);
      run += __shfl_sync(WARP_FULL, incl, 31);
    }
  }
  if (lane == 0) {
    d.world_pairadr[w] = adr < 0 ? 0 : adr;
    d.world_npair[w] = total;
  }
  __syncwarp();
}

// The reference's broadphase choice (collision_driver.py:537-540): nxn for ngeom <= 100, else
// sweep-and-prune (which needs sap_smem_floats(ngeom) floats of warp scratch `sm`).
__device__ __forceinline__ bool use_sap(const MjbModel& m) { return m.ngeom > 100; }

struct ContactOut {
  const MjbModel* m;
  const MjbData* d;
  int w, g1, g2;
  int next;  // next contact index to write, or < 0 to only count
  int count;
  float margin;
  // collision_primitive.py:52-70 + get_contact_solver_params_kernel (collision_driver.py:304-347)
  __device__ void add(float dist, f3 pos, const m33& frame) {
    if (!((dist - margin) < 0.f)) return;
    count++;
    if (next < 0) return;
    const int k = next++;
    const MjbModel& M = *m;
    const MjbData& D = *d;
    D.contact_dist[k] = dist;
    st3(D.contact_pos + 3 * k, pos);
    st9(D.contact_frame + 9 * k, frame);
    D.contact_geom[2 * k] = g1;
    D.contact_geom[2 * k + 1] = g2;
    D.contact_worldid[k] = w;
    const float gap = fmaxf(M.geom_gap[g1], M.geom_gap[g2]);
    const float sm1 = M.geom_solmix[g1], sm2 = M.geom_solmix[g2];
    float mix = sm1 / (sm1 + sm2);
    if (sm1 < kMinVal && sm2 < kMinVal) mix = 0.5f;
    else if (sm1 < kMinVal) mix = 0.f;
    else if (sm2 < kMinVal) mix = 1.f;
    const int p1 = M.geom_priority[g1], p2 = M.geom_priority[g2];
    if (p1 != p2) mix = p1 > p2 ? 1.f : 0.f;
    const int c1 = M.geom_condim[g1], c2 = M.geom_condim[g2];
    D.contact_dim[k] = p1 == p2 ? max(c1, c2) : (p1 > p2 ? c1 : c2);
    const float* r1 = M.geom_solref + 2 * g1;
    const float* r2 = M.geom_solref + 2 * g2;
    if (r1[0] > 0.f && r2[0] > 0.f) {
      D.contact_solref[2 * k] = mix * r1[0] + (1.f - mix) * r2[0];
      D.contact_solref[2 * k + 1] = mix * r1[1] + (1.f - mix) * r2[1];
    } else {
      D.contact_solref[2 * k] = fminf(r1[0], r2[0]);
      D.contact_solref[2 * k + 1] = fminf(r1[1], r2[1]);
    }
    if (D.contact_solreffriction) {
      D.contact_solreffriction[2 * k] = 0.f;
      D.contact_solreffriction[2 * k + 1] = 0.f;
    }
    D.contact_includemargin[k] = margin - gap;
    const float f0 = fmaxf(M.geom_friction[3 * g1], M.geom_friction[3 * g2]);
    const float f1 = fmaxf(M.geom_friction[3 * g1 + 1], M.geom_friction[3 * g2 + 1]);
    const float f2 = fmaxf(M.geom_friction[3 * g1 + 2], M.geom_friction[3 * g2 + 2]);
    float* fr = D.contact_friction + 5 * k;
    fr[0] = f0; fr[1] = f0; fr[2] = f1; fr[3] = f2; fr[4] = f2;
    for (int i = 0; i < 5; i++)
      D.contact_solimp[5 * k + i] = mix * M.geom_solimp[5 * g1 + i] + (1.f - mix) * M.geom_solimp[5 * g2 + i];
  }
};

__device__ __forceinline__ void plane_sphere_raw(f3 n, f3 ppos, f3 spos, float r, float& dist, f3& pos) {
  dist = dot(spos - ppos, n) - r;
  pos = spos - n * (r + 0.5f * dist);
}

__device__ __forceinline__ void sphere_sphere_raw(ContactOut& o, f3 p1, float r1, f3 p2, float r2) {
  const f3 dir = p2 - p1;
  float dist = length(dir);
  const f3 n = dist == 0.f ? mk3(1.f, 0.f, 0.f) : dir * (1.f / dist);
  dist = dist - (r1 + r2);
  const f3 pos = p1 + n * (r1 + 0.5f * dist);
  o.add(dist, pos, make_frame(n));
}

// collision_primitive.py:235-268 for one candidate pair
__device__ void narrow_pair(ContactOut& o) {
  const MjbModel& m = *o.m;
  const int g1 = o.g1, g2 = o.g2, w = o.w;
  const float* gxpos = o.d->geom_xpos + W(w, 3 * m.ngeom);
  const float* gxmat = o.d->geom_xmat + W(w, 9 * m.ngeom);
  const int t1 = m.geom_type[g1], t2 = m.geom_type[g2];
  const f3 pos1 = ld3(gxpos + 3 * g1), pos2 = ld3(gxpos + 3 * g2);
  const m33 r1 = ld9(gxmat + 9 * g1), r2 = ld9(gxmat + 9 * g2);
  const f3 n1 = col(r1, 2);
  const f3 sz1 = ld3(m.geom_size + 3 * g1), sz2 = ld3(m.geom_size + 3 * g2);
  if (t1 == GEOM_PLANE && t2 == GEOM_SPHERE) {  // :73-93
    float dist;
    f3 pos;
    plane_sphere_raw(n1, pos1, pos2, sz2.x, dist, pos);
    o.add(dist, pos, make_frame(n1));
  } else if (t1 == GEOM_SPHERE && t2 == GEOM_SPHERE) {  // :96-137
    sphere_sphere_raw(o, pos1, sz1.x, pos2, sz2.x);
  } else if (t1 == GEOM_PLANE && t2 == GEOM_CAPSULE) {  // :166-195
    const f3 n = n1, axis = col(r2, 2);
    const f3 bv = axis - n * dot(n, axis);
    const float bn = length(bv);
    f3 b = bn == 0.f ? bv : bv * (1.f / bn);
    if (bn < 0.5f) b = (-0.5f < n.y && n.y < 0.5f) ? mk3(0.f, 1.f, 0.f) : mk3(0.f, 0.f, 1.f);
    const f3 c = cross(n, b);
    const m33 frame{{n.x, n.y, n.z, b.x, b.y, b.z, c.x, c.y, c.z}};
    const f3 seg = axis * sz2.y;
    float dist;
    f3 pos;
    plane_sphere_raw(n, pos1, pos2 + seg, sz2.x, dist, pos);
    o.add(dist, pos, frame);
    plane_sphere_raw(n, pos1, pos2 - seg, sz2.x, dist, pos);
    o.add(dist, pos, frame);
  } else if (t1 == GEOM_PLANE && t2 == GEOM_BOX) {  // :198-232
    int cnt = 0;
    const float dist = dot(pos2 - pos1, n1);
    const m33 frame = make_frame(n1);
    for (int i = 0; i < 8; i++) {
      f3 corner = mk3((i & 1) ? sz2.x : -sz2.x, (i & 2) ? sz2.y : -sz2.y, (i & 4) ? sz2.z : -sz2.z);
      corner = mulmv(r2, corner);
      const float ldist = dot(n1, corner);
      if (dist + ldist > o.margin || ldist > 0.f) continue;
      const float cdist = dist + ldist;
      o.add(cdist, corner + pos2 + n1 * (cdist / -2.f), frame);
      if (++cnt >= 4) break;
    }
  } else if (t1 == GEOM_CAPSULE && t2 == GEOM_CAPSULE) {  // :140-163
    const f3 s1 = col(r1, 2) * sz1.y, s2 = col(r2, 2) * sz2.y;
    f3 pa, pb;
    closest_segment_to_segment_points(pos1 - s1, pos1 + s1, pos2 - s2, pos2 + s2, pa, pb);
    sphere_sphere_raw(o, pa, sz1.x, pb, sz2.x);
  }
}

__device__ __forceinline__ ContactOut make_out(const MjbModel& m, const MjbData& d, int w, int pair) {
  ContactOut o;
  o.m = &m;
  o.d = &d;
  o.w = w;
  o.g1 = d.collision_pair[2 * pair];
  o.g2 = d.collision_pair[2 * pair + 1];
  o.next = -1;
  o.count = 0;
  o.margin = fmaxf(m.geom_margin[o.g1], m.geom_margin[o.g2]);
  return o;
}

// Pairs whose contact count (at most 4: plane-box) a lane keeps from the counting pass, 3 bits
// each in one 64-bit register: the first kCountChunks chunks of 32 pairs (672 pairs per world).
// The write pass evaluates only those pairs that make contacts; pairs beyond are counted again.
constexpr int kCountChunks = 21;

// collision_primitive.py:271-274 over this world's pairs.  The world's contacts take one
// contiguous block: a counting pass sizes it, a write pass fills it in pair order.
__device__ void primitive_narrowphase(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int pa = d.world_pairadr[w], np = d.world_npair[w];
  int total = 0;
  unsigned long long counts = 0;
  for (int base = 0, chunk = 0; base < np; base += 32, chunk++) {
    int c = 0;
    if (base + lane < np) {
      ContactOut o = make_out(m, d, w, pa + base + lane);
      narrow_pair(o);
      c = o.count;
    }
    if (chunk < kCountChunks) counts |= (unsigned long long)c << (3 * chunk);
    total += warp_sum_i(c);
  }
  const int adr = reserve(d.ncon, total, d.nconmax, d.world_status ? d.world_status + w : nullptr,
                          MJB_WS_CONTACT_OVERFLOW, lane);
  if (adr < 0) total = 0;
  if (total > 0) {
    int run = 0;
    for (int base = 0, chunk = 0; base < np; base += 32, chunk++) {
      int c = 0;
      if (chunk < kCountChunks) {
        c = (int)((counts >> (3 * chunk)) & 7ull);
      } else if (base + lane < np) {
        ContactOut o = make_out(m, d, w, pa + base + lane);
        narrow_pair(o);
        c = o.count;
      }
      int tot;
      const int off = warp_excl_scan(c, lane, &tot);
      if (c > 0) {
        ContactOut o = make_out(m, d, w, pa + base + lane);
        o.next = adr + run + off;
        narrow_pair(o);
      }
      run += tot;
    }
  }
  if (lane == 0) {
    d.world_conadr[w] = adr < 0 ? 0 : adr;
    d.world_ncon[w] = total;
  }
  __syncwarp();
}

// collision_driver.py:525-547 (ngeom <= 100 path; larger models go through sap_broadphase, whose
// pair set is the same set of overlapping candidates)
// sm: sap_smem_floats(ngeom) floats of warp scratch when use_sap(m)
__device__ void collision(const MjbModel& m, const MjbData& d, int w, int lane, float* sm) {
  if (use_sap(m)) sap_broadphase(m, d, w, lane, sm);
  else nxn_broadphase(m, d, w, lane);
  primitive_narrowphase(m, d, w, lane);
}

// ------------------------------------------------------------------------------------------
// constraint.py:22-73
__device__ void update_efc_row(const MjbModel& m, const MjbData& d, int r, float pos_aref,
                               float pos_imp, float invweight, const float* solref,
                               const float* solimp, float margin, bool refsafe, float Jqvel) {
  float timeconst = solref[0], dampratio = solref[1];
  float dmin = solimp[0], dmax = solimp[1], width = solimp[2], mid = solimp[3], power = solimp[4];
  if (refsafe) timeconst = fmaxf(timeconst, 2.f * m.timestep);
  dmin = fminf(fmaxf(dmin, kMinImp), kMaxImp);
  dmax = fminf(fmaxf(dmax, kMinImp), kMaxImp);
  width = fmaxf(kMinVal, width);
  mid = fminf(fmaxf(mid, kMinImp), kMaxImp);
  power = fmaxf(1.f, power);
  float k = 1.f / (dmax * dmax * timeconst * timeconst * dampratio * dampratio);
  float b = 2.f / (dmax * timeconst);
  if (solref[0] <= 0.f) k = -solref[0] / (dmax * dmax);
  if (solref[1] <= 0.f) b = -solref[1] / dmax;
  const float imp_x = fabsf(pos_imp) / width;
  float imp;
  if (imp_x > 1.f) {
    imp = dmax;
  } else {
    float imp_y;
    if (imp_x < mid) imp_y = (1.f / powf(mid, power - 1.f)) * powf(imp_x, power);
    else imp_y = 1.f - (1.f / powf(1.f - mid, power - 1.f)) * powf(1.f - imp_x, power);
    imp = dmin + imp_y * (dmax - dmin);
    imp = fminf(fmaxf(imp, dmin), dmax);
  }
  d.efc_D[r] = 1.f / fmaxf(invweight * (1.f - imp) / imp, kMinVal);
  d.efc_aref[r] = -k * imp * pos_aref - b * Jqvel;
  d.efc_pos[r] = pos_aref + margin;
  d.efc_margin[r] = margin;
}

// constraint.py:213-240: joint limits (:104-141), then condim-3 pyramidal contacts (:144-210)
__device__ void make_constraint(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nv = m.nv;
  const bool on = !(m.disableflags & DSBL_CONSTRAINT);
  const bool do_lim = on && !(m.disableflags & DSBL_LIMIT) && m.nlimit > 0;
  const bool do_con = on && !(m.disableflags & DSBL_CONTACT) && m.cone == 0;
  const bool refsafe = !(m.disableflags & DSBL_REFSAFE);
  const float* qpos = d.qpos + W(w, m.nq);
  const float* qvel = d.qvel + W(w, nv);
  const int ca = d.world_conadr[w], nc = d.world_ncon[w];
  int nlim = 0, ncact = 0;
  if (do_lim) {
    for (int base = 0; base < m.nlimit; base += 32) {
      const int l = base + lane;
      bool act = false;
      if (l < m.nlimit) {
        const int j = m.jnt_limited_slide_hinge_adr[l];
        const float q = qpos[m.jnt_qposadr[j]];
        act = (fminf(q - m.jnt_range[2 * j], m.jnt_range[2 * j + 1] - q) - m.jnt_margin[j]) < 0.f;
      }
      nlim += __popc(__ballot_sync(WARP_FULL, act));
    }
  }
  if (do_con) {
    for (int base = 0; base < nc; base += 32) {
      const int c = ca + base + lane;
      const bool act = base + lane < nc && d.contact_dim[c] == 3 &&
                       (d.contact_dist[c] - d.contact_includemargin[c]) < 0.f;
      ncact += __popc(__ballot_sync(WARP_FULL, act));
    }
  }
  int n = nlim + 4 * ncact;
  const int adr = reserve(d.nefc, n, d.njmax, d.world_status ? d.world_status + w : nullptr,
                          MJB_WS_EFC_OVERFLOW, lane);
  if (adr < 0) n = 0;
  if (lane == 0) {
    d.world_efcadr[w] = adr < 0 ? 0 : adr;
    d.world_nefc[w] = n;
  }
  if (n == 0) {
    __syncwarp();
    return;
  }
  // limit rows
  if (nlim > 0) {
    for (int e = lane; e < nlim * nv; e += 32) d.efc_J[size_t(adr) * nv + e] = 0.f;
    __syncwarp();
    int run = 0;
    for (int base = 0; base < m.nlimit; base += 32) {
      const int l = base + lane;
      bool act = false;
      float q = 0.f, dmin = 0.f, dmax = 0.f, pos = 0.f;
      int j = 0;
      if (l < m.nlimit) {
        j = m.jnt_limited_slide_hinge_adr[l];
        q = qpos[m.jnt_qposadr[j]];
        dmin = q - m.jnt_range[2 * j];
        dmax = m.jnt_range[2 * j + 1] - q;
        pos = fminf(dmin, dmax) - m.jnt_margin[j];
        act = pos < 0.f;
      }
      const unsigned mask = __ballot_sync(WARP_FULL, act);
      if (act) {
        const int r = adr + run + __popc(mask & ((1u << lane) - 1u));
        const int dof = m.jnt_dofadr[j];
        const float J = float(dmin < dmax) * 2.f - 1.f;
        d.efc_J[size_t(r) * nv + dof] = J;
        d.efc_worldid[r] = w;
        update_efc_row(m, d, r, pos, pos, m.dof_invweight0[dof], m.jnt_solref + 2 * j,
                       m.jnt_solimp + 5 * j, m.jnt_margin[j], refsafe, J * qvel[dof]);
      }
      run += __popc(mask);
    }
  }
  // contact rows: lanes over dofs build the 4 pyramid rows of one contact at a time
  if (ncact > 0) {
    const float* cdof = d.cdof + W(w, 6 * nv);
    const float* sc = d.subtree_com + W(w, 3 * m.nbody);
    int r = adr + nlim;
    for (int k = 0; k < nc; k++) {
      const int c = ca + k;
      if (!(d.contact_dim[c] == 3 && (d.contact_dist[c] - d.contact_includemargin[c]) < 0.f)) continue;
      const float pos = d.contact_dist[c] - d.contact_includemargin[c];
      const int b1 = m.geom_bodyid[d.contact_geom[2 * c]], b2 = m.geom_bodyid[d.contact_geom[2 * c + 1]];
      const float* fr = d.contact_frame + 9 * c;
      const float* fri = d.contact_friction + 5 * c;
      const f3 cp = ld3(d.contact_pos + 3 * c);
      const f3 off1 = cp - ld3(sc + 3 * m.body_rootid[b1]);
      const f3 off2 = cp - ld3(sc + 3 * m.body_rootid[b2]);
      float jq[4] = {0.f, 0.f, 0.f, 0.f};
      for (int i = lane; i < nv; i += 32) {
        const s6 cd = ld6(cdof + 6 * i);
        const f3 ang{cd.v[0], cd.v[1], cd.v[2]}, lin{cd.v[3], cd.v[4], cd.v[5]};
        const int db = m.dof_bodyid[i];
        // constraint.py:76-101: the dof moves body b iff its body is an ancestor-or-self of b
        const float in1 = (db != 0 && db <= b1 && b1 < m.body_subtreeend[db]) ? 1.f : 0.f;
        const float in2 = (db != 0 && db <= b2 && b2 < m.body_subtreeend[db]) ? 1.f : 0.f;
        const f3 j1 = (lin + cross(ang, off1)) * in1;
        const f3 j2 = (lin + cross(ang, off2)) * in2;
        const f3 jd = j2 - j1;
        const float diff0 = fr[0] * jd.x + fr[1] * jd.y + fr[2] * jd.z;
        const float diff1 = fr[3] * jd.x + fr[4] * jd.y + fr[5] * jd.z;
        const float diff2 = fr[6] * jd.x + fr[7] * jd.y + fr[8] * jd.z;
        const float Jr[4] = {diff0 + diff1 * fri[0], diff0 - diff1 * fri[0], diff0 + diff2 * fri[1],
                             diff0 - diff2 * fri[1]};
#pragma unroll
        for (int e = 0; e < 4; e++) {
          d.efc_J[size_t(r + e) * nv + i] = Jr[e];
          jq[e] += Jr[e] * qvel[i];
        }
      }
#pragma unroll
      for (int e = 0; e < 4; e++) jq[e] = warp_sum(jq[e]);
      if (lane < 4) {
        const float fri0 = fri[0];
        float invweight = m.body_invweight0[2 * b1] + m.body_invweight0[2 * b2];
        invweight = invweight + fri0 * fri0 * invweight;
        invweight = invweight * 2.f * fri0 * fri0 / m.impratio;
        const float jql = lane == 0 ? jq[0] : (lane == 1 ? jq[1] : (lane == 2 ? jq[2] : jq[3]));
        d.efc_worldid[r + lane] = w;
        update_efc_row(m, d, r + lane, pos, pos, invweight, d.contact_solref + 2 * c,
                       d.contact_solimp + 5 * c, d.contact_includemargin[c], refsafe, jql);
      }
      r += 4;
    }
  }
  __syncwarp();
}

}  // namespace mjb
