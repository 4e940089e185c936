// hb_pairs.cuh -- the FP32 2nd-order step kernel with two cells per lane.
//
// Included by hb_fused.cu inside its anonymous namespace (it uses that file's
// TilePartial, BcTable, close_group, mbarrier/TMA helpers and RowsView-style
// indexing).  Same scheme, decisions and data layout as rows_step_kernel
// (HC/flucCal_2ndOrder_jh_improved_Kernel.cu:43-506 per face,
// HC/friction_implicit_andUpdate_jh_Kernel.cu:22-146 and
// HC/timeControl_Kernel.cu:164-198 per cell, HC/fluxMaskGenerator_Kernel.cu:19-42
// for the activity rule), laid out for the FP32 pipes of sm_100:
//  * a CTA of 4 warps owns a tile of 64 columns x TY rows; lane j of a warp
//    owns the horizontal cell pair (2j, 2j+1) and walks TY/4 rows;
//  * every face is evaluated once, by a function that computes TWO faces in
//    the two halves of packed f32x2 registers: per row a lane evaluates the
//    west faces of its two cells (2j-1|2j and 2j|2j+1) and their two south
//    faces, so every add, multiply and FMA of the MUSCL edges, hydrostatic
//    reconstruction, HLLC solver and bed-slope terms issues once for two
//    faces (add/sub/mul/fma.rn.ftz.f32x2); compares, selects, min/max and
//    the special functions stay per face;
//  * the east face of cell 2j is the lane's own second west face; that of
//    cell 2j+1 comes from lane j+1 by one shuffle per value (lane 31: a
//    tile-edge pre-pass), so shuffles and loop overhead are per cell pair;
//  * the cell update (activity, rain, implicit friction, h_max, CFL speed,
//    FP64 volume) runs on the pair, packed where the arithmetic allows;
//  * a step is one launch of pairs_mixed_kernel, one CTA per tile over the
//    prepared list (general tiles with a valid cell, all-valid tiles, tiles
//    without a valid cell), every CTA at the all-valid build's register cap;
//    pairs_step_kernel keeps the general and all-valid builds as two launches
//    for a 3-CTA register cap or a looping grid.
// Every packed operation is pinned by inline PTX (no contraction freedom), and
// all faces -- interior, tile-edge and ghost -- go through the same packed
// function, so a face evaluated by two tiles, or by the general and the
// all-valid build, comes out bit for bit the same, and a state symmetric
// about a wall stays symmetric.

// ---------------------------------------------------------------------------
// Packed and pinned FP32 arithmetic
// ---------------------------------------------------------------------------
using f2 = float2;

__device__ __forceinline__ f2 pk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ f2 dup(float a) { return make_float2(a, a); }

__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 r;
  asm("{.reg .b64 A, B, D;\n\tmov.b64 A, {%2, %3};\n\tmov.b64 B, {%4, %5};\n\t"
      "add.rn.ftz.f32x2 D, A, B;\n\tmov.b64 {%0, %1}, D;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 r;
  asm("{.reg .b64 A, B, D;\n\tmov.b64 A, {%2, %3};\n\tmov.b64 B, {%4, %5};\n\t"
      "sub.rn.ftz.f32x2 D, A, B;\n\tmov.b64 {%0, %1}, D;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 r;
  asm("{.reg .b64 A, B, D;\n\tmov.b64 A, {%2, %3};\n\tmov.b64 B, {%4, %5};\n\t"
      "mul.rn.ftz.f32x2 D, A, B;\n\tmov.b64 {%0, %1}, D;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
// a * b + c, one rounding
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 r;
  asm("{.reg .b64 A, B, C, D;\n\tmov.b64 A, {%2, %3};\n\tmov.b64 B, {%4, %5};\n\t"
      "mov.b64 C, {%6, %7};\n\tfma.rn.ftz.f32x2 D, A, B, C;\n\tmov.b64 {%0, %1}, D;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return r;
}
// scalar form, used where a value is formed for one cell only (x-slopes)
__device__ __forceinline__ float sub1(float a, float b) {
  float r;
  asm("sub.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
// approximate reciprocal, square root, base-2 logarithm and exponential (the
// hardware's special-function unit, as the -prec-div/-prec-sqrt=false build
// of the 32-wide kernel uses)
__device__ __forceinline__ float rcpa(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sqrta(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float lg2a(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2a(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

constexpr float kHsF = 1.0e-6f;          // h_small
constexpr float kGF = 9.81f;             // g
constexpr float kHalfGF = 0.5f * 9.81f;  // exact: a power-of-two scaling of g

// minmod(d1, d2) (HC/flucCal_2ndOrder_jh_improved_Kernel.cu:74-81): 0 when
// the signs differ, else the one of smaller magnitude.  The reference tests
// the sign of d1 * d2 in FP64; formed by min and max here (four ALU
// operations, no product), so differences below 1e-19, whose FP32 product
// would flush to zero, keep their sign test too.
__device__ __forceinline__ float mmod(float d1, float d2) {
  return fmaxf(fminf(d1, d2), fminf(0.f, fmaxf(d1, d2)));
}
// slope of c between its minus-side neighbour m and plus-side neighbour p
// (x-slopes: one cell at a time)
__device__ __forceinline__ float slope1(float c, float m, float p) {
  return mmod(sub1(c, m), sub1(p, c));
}
// the same for a vertical pair of cells (y-slopes)
__device__ __forceinline__ f2 slope2(f2 c, f2 m, f2 p) {
  const f2 d1 = sub2(c, m), d2 = sub2(p, c);
  return pk(mmod(d1.x, d2.x), mmod(d1.y, d2.y));
}

struct Cel2 {
  f2 h, qx, qy, z;
};
struct Slp2 {
  f2 h, z, qx, qy;
};
// two faces: mass flux, x- and y-momentum flux (global frame, from the
// west/south side A), bed-slope terms of side A and side B
struct Fc2 {
  f2 fh, fx, fy, sa, sb;
};

// Two faces in the face frame.  Inputs with beds measured from the minus
// cell's bed: the edge states L (minus side) and R (plus side) -- depth, bed,
// normal and tangential discharge -- the two cells' depths ah, bh and the
// plus cell's bed bz.  Velocities are taken from the edge states, then the
// hydrostatic step (HC/flucCal_2ndOrder_jh_improved_Kernel.cu:43-72), the HLLC
// flux (:109-195, with the single-precision shortcuts of hllc<float, true>)
// and the two bed-slope terms (:494-501).  fn / ft: normal / tangential
// momentum flux; ft is linear in the tangential discharge, so a caller that
// passes +q instead of -q for it takes -ft.
//
// ORDER 2 raises the downhill edge level to the other's (the 2nd-order
// hydrostatic step, :43-72); ORDER 1 averages the two edge levels when their
// ordering is the reverse of the cells' (the 1st-order step,
// HC/fluxCal_jh_modified_surface_Kernel.cu:96-139).
//
// The hydrostatic step runs with beds measured from the higher of the two edge
// beds, o = max(Lz, Rz) (every operation of the scheme is invariant under a
// common shift of z).  The upper edge then has bed 0 and its free surface is
// its depth exactly, so a film of a few h_small on a bump keeps its depth to
// the last bit instead of being rounded at the scale of the bed step (6e-8 m
// per 0.5 m of relief in FP32), which decided which side of h_small such a
// cell fell on.
//
// The edge discharges enter only through the edge velocities, so a dry cell's
// zero edge discharge is applied there: the velocity factor of an edge is 0
// when its depth or its cell's depth is below h_small.  dd0 / dd1: the two
// cells of that face are both dry; its fluxes are zero (with those of a face
// whose reconstructed depths are both below h_small).
template <int ORDER>
__device__ __forceinline__ void face_core2(f2 ah, f2 bh, f2 bz, f2 Lh, f2 Lz0, f2 Lqn, f2 Lqt,
                                           f2 Rh, f2 Rz0, f2 Rqn, f2 Rqt, f2 &fh, f2 &fn,
                                           f2 &ft, f2 &sa, f2 &sb, bool dd0 = false,
                                           bool dd1 = false) {
  const f2 o = pk(fmaxf(Lz0.x, Rz0.x), fmaxf(Lz0.y, Rz0.y));
  const f2 Lz = sub2(Lz0, o), Rz = sub2(Rz0, o);   // one of the two is exactly 0
  const f2 bzo = sub2(bz, o);                       // the plus cell's bed
  const f2 wa = sub2(ah, o), wb = add2(bzo, bh);    // the cells' free surfaces
  // velocities of the edge states
  const f2 il = pk(Lh.x < kHsF || ah.x < kHsF ? 0.f : rcpa(Lh.x),
                   Lh.y < kHsF || ah.y < kHsF ? 0.f : rcpa(Lh.y));
  const f2 ir = pk(Rh.x < kHsF || bh.x < kHsF ? 0.f : rcpa(Rh.x),
                   Rh.y < kHsF || bh.y < kHsF ? 0.f : rcpa(Rh.y));
  const f2 uL = mul2(Lqn, il), vL = mul2(Lqt, il);
  const f2 uR = mul2(Rqn, ir), vR = mul2(Rqt, ir);
  // hydrostatic reconstruction
  f2 Lw = add2(Lh, Lz), Rw = add2(Rh, Rz);
  {
    const float hix = fmaxf(wa.x, wb.x), lox = fminf(wa.x, wb.x);
    const float hiy = fmaxf(wa.y, wb.y), loy = fminf(wa.y, wb.y);
    Lw = pk(fmaxf(fminf(Lw.x, hix), lox), fmaxf(fminf(Lw.y, hiy), loy));
    Rw = pk(fmaxf(fminf(Rw.x, hix), lox), fmaxf(fminf(Rw.y, hiy), loy));
    if constexpr (ORDER == 2) {
      const float mx = fmaxf(Lw.x, Rw.x), my = fmaxf(Lw.y, Rw.y);
      if (wa.x > wb.x) Lw.x = mx; else Rw.x = mx;
      if (wa.y > wb.y) Lw.y = my; else Rw.y = my;
    } else {
      const f2 flip = mul2(sub2(wa, wb), sub2(Lw, Rw));
      const f2 avg = mul2(add2(Lw, Rw), dup(0.5f));
      if (flip.x < 0.f) Lw.x = Rw.x = avg.x;
      if (flip.y < 0.f) Lw.y = Rw.y = avg.y;
    }
  }
  const f2 Lz1 = sub2(Lw, Lh), Rz1 = sub2(Rw, Rh);
  const f2 zbm = pk(fmaxf(Lz1.x, Rz1.x), fmaxf(Lz1.y, Rz1.y));
  const f2 Ld = sub2(Lw, zbm), Rd = sub2(Rw, zbm);
  const f2 hL = pk(fmaxf(Ld.x, 0.f), fmaxf(Ld.y, 0.f));
  const f2 hR = pk(fmaxf(Rd.x, 0.f), fmaxf(Rd.y, 0.f));
  const f2 zL = sub2(Lw, hL), zR = sub2(Rw, hR);
  // bed-slope terms of both sides
  sa = mul2(mul2(dup(kHalfGF), add2(ah, hL)), add2(zL, o));  // zL - (the minus cell's bed, -o)
  sb = mul2(mul2(dup(kHalfGF), add2(bh, hR)), sub2(zR, bzo));
  // HLLC
  const f2 qnL = mul2(uL, hL), qnR = mul2(uR, hR);
  const f2 gL = mul2(dup(kGF), hL), gR = mul2(dup(kGF), hR);
  const f2 aL = pk(sqrta(gL.x), sqrta(gL.y)), aR = pk(sqrta(gR.x), sqrta(gR.y));
  const f2 base = fma2(add2(aL, aR), dup(0.5f), mul2(sub2(uL, uR), dup(0.25f)));
  const f2 ustar = sub2(fma2(add2(uL, uR), dup(0.5f), aL), aR);
  const f2 astar = pk(fabsf(base.x), fabsf(base.y));
  const f2 t1 = fma2(dup(-2.f), aR, uR), t2 = sub2(uL, aL), t3 = sub2(ustar, astar);
  const f2 t4 = fma2(dup(2.f), aL, uL), t5 = add2(uR, aR), t6 = add2(ustar, astar);
  const f2 sL = pk(hL.x <= kHsF ? t1.x : fminf(t2.x, t3.x), hL.y <= kHsF ? t1.y : fminf(t2.y, t3.y));
  const f2 sR = pk(hR.x <= kHsF ? t4.x : fmaxf(t5.x, t6.x), hR.y <= kHsF ? t4.y : fmaxf(t5.y, t6.y));
  const f2 hfL = qnL, hfR = qnR;
  const f2 nfL = fma2(uL, qnL, mul2(mul2(dup(kHalfGF), hL), hL));
  const f2 nfR = fma2(uR, qnR, mul2(mul2(dup(kHalfGF), hR), hR));
  const f2 pR = mul2(hR, sub2(uR, sR)), pL = mul2(hL, sub2(uL, sL));
  const f2 num = sub2(mul2(sL, pR), mul2(sR, pL)), den = sub2(pR, pL);
  const f2 sM = mul2(num, pk(rcpa(den.x), rcpa(den.y)));
  const f2 dS = sub2(sR, sL);
  const f2 inv = pk(rcpa(dS.x), rcpa(dS.y));
  const f2 sLR = mul2(sL, sR);
  const f2 hfM = mul2(fma2(sLR, sub2(hR, hL), sub2(mul2(sR, hfL), mul2(sL, hfR))), inv);
  f2 vU;
  const f2 nfM = mul2(fma2(sLR, sub2(qnR, qnL), sub2(mul2(sR, nfL), mul2(sL, nfR))), inv);
#pragma unroll
  for (int c = 0; c < 2; c++) {
    const float sl = c ? sL.y : sL.x, sr = c ? sR.y : sR.x, sm = c ? sM.y : sM.x;
    // the reference's chain sL >= 0 / sL < 0 <= sM / sM < 0 <= sR / else,
    // with sL finite (it is, for a finite state)
    const bool left = 0.f <= sl;
    const bool midL = !left && 0.f <= sm;
    const bool midR = !left && sm < 0.f && 0.f <= sr;
    const bool mid = midL || midR;
    const bool dry = ((c ? hL.y : hL.x) < kHsF && (c ? hR.y : hR.x) < kHsF) || (c ? dd1 : dd0);
    float h_ = left ? (c ? hfL.y : hfL.x) : (mid ? (c ? hfM.y : hfM.x) : (c ? hfR.y : hfR.x));
    float n_ = left ? (c ? nfL.y : nfL.x) : (mid ? (c ? nfM.y : nfM.x) : (c ? nfR.y : nfR.x));
    if (dry) h_ = n_ = 0.f;
    // the tangential flux is the mass flux times the upwind side's
    // tangential velocity in every region (the reference forms the
    // unstarred ones as u * (v * h); (u * h) * v here: one rounding apart)
    const float vu = (left || midL) ? (c ? vL.y : vL.x) : (c ? vR.y : vR.x);
    if (c) {
      fh.y = h_; fn.y = n_; vU.y = vu;
    } else {
      fh.x = h_; fn.x = n_; vU.x = vu;
    }
  }
  ft = mul2(fh, vU);
}

// Two interior faces between valid cells A (minus side: west, or south) and
// B (plus side) along DIR (0: normal +x; 1: normal +y, towards the row
// above), from the cells and their minmod slopes along DIR.  ORDER 2: MUSCL
// edge states (HC/flucCal_2ndOrder_jh_improved_Kernel.cu:83-107, 410-485);
// ORDER 1: the cells themselves, only the bed taking half its slope on a side
// whose neighbour across the face is wet
// (HC/fluxCal_jh_modified_surface_Kernel.cu:577-593; only sA.z, sB.z are
// read).  The frame measures beds from A's bed.  A face whose two cells are
// both dry is zero.
template <int DIR, int ORDER = 2>
__device__ __forceinline__ Fc2 face2(const Cel2 &A, const Cel2 &B, const Slp2 &sA,
                                     const Slp2 &sB) {
  Fc2 o;
  const bool dd0 = A.h.x < kHsF && B.h.x < kHsF, dd1 = A.h.y < kHsF && B.h.y < kHsF;
  // no early return when both faces are dry: one branch-free block lets the
  // compiler interleave a row's x- and y-faces (the dry faces are zeroed in
  // face_core2 and below)
  const f2 bz = sub2(B.z, A.z);
  f2 Lh, Lz, Lqx, Lqy, Rh, Rz, Rqx, Rqy;
  if constexpr (ORDER == 2) {
    Lh = fma2(dup(0.5f), sA.h, A.h);
    Lz = mul2(dup(0.5f), sA.z);
    Lqx = fma2(dup(0.5f), sA.qx, A.qx);
    Lqy = fma2(dup(0.5f), sA.qy, A.qy);
    Rh = fma2(dup(-0.5f), sB.h, B.h);
    Rz = fma2(dup(-0.5f), sB.z, bz);
    Rqx = fma2(dup(-0.5f), sB.qx, B.qx);
    Rqy = fma2(dup(-0.5f), sB.qy, B.qy);
    // a dry cell's edges carry no discharge: face_core2 takes their
    // velocities as 0
  } else {
    Lh = A.h;
    Rh = B.h;
    Lqx = A.qx;
    Lqy = A.qy;
    Rqx = B.qx;
    Rqy = B.qy;
    const f2 lz = mul2(dup(0.5f), sA.z), rz = fma2(dup(-0.5f), sB.z, bz);
    Lz = pk(B.h.x > kHsF ? lz.x : 0.f, B.h.y > kHsF ? lz.y : 0.f);
    Rz = pk(A.h.x > kHsF ? rz.x : bz.x, A.h.y > kHsF ? rz.y : bz.y);
  }
  f2 fn, ft;
  if constexpr (DIR == 0) {
    face_core2<ORDER>(A.h, B.h, bz, Lh, Lz, Lqx, Lqy, Rh, Rz, Rqx, Rqy, o.fh, fn, ft, o.sa,
                      o.sb, dd0, dd1);
    o.fx = fn;
    o.fy = ft;
  } else {
    // normal +y, tangent -x: the tangential discharge is passed as +qx, so
    // the face's x-momentum flux (-ft of the -qx form) is ft
    face_core2<ORDER>(A.h, B.h, bz, Lh, Lz, Lqy, Lqx, Rh, Rz, Rqy, Rqx, o.fh, fn, ft, o.sa,
                      o.sb, dd0, dd1);
    o.fx = ft;
    o.fy = fn;
  }
  if (dd0) o.sa.x = o.sb.x = 0.f;  // the fluxes: face_core2
  if (dd1) o.sa.y = o.sb.y = 0.f;
  return o;
}

// Face between valid cell C and the ghost of its missing neighbour on `side`
// (0 E, 1 N, 2 W, 3 S), built from C's boundary class
// (HC/flucCal_2ndOrder_jh_improved_Kernel.cu:197-332): no reconstruction, C
// evaluated as the minus side in its outward frame, the same packed face
// function (one face, duplicated).  Result in the face convention of the
// tile (flux from the west/south side of the face) and C's bed-slope term.
struct Ghost1 {
  float fh, fx, fy, sc;
};
template <int ORDER>
__device__ __noinline__ Ghost1 ghost_face1(float ch, float cqx, float cqy, float cz, int type,
                                           const double *bcv, float datum, int side) {
  Ghost1 r{0.f, 0.f, 0.f, 0.f};
  const float n0 = side == 0 ? 1.f : (side == 2 ? -1.f : 0.f);
  const float n1 = side == 1 ? 1.f : (side == 3 ? -1.f : 0.f);
  Cell<float> Cl, G;
  Cl.h = ch;
  Cl.qx = cqx;
  Cl.qy = cqy;
  Cl.z = 0.f;  // beds measured from C's bed
  Cl.wl = ch;
  const float hb = (float)bcv[0];
  const float wlb = (float)(bcv[1] - (double)datum) - cz;
  const float qxb = (float)bcv[2], qyb = (float)bcv[3];
  // FALL (type 9) is a ghost of the 1st-order scheme only
  if (!ghost(type, ORDER == 1, Cl, n0, n1, hb, wlb, qxb, qyb, G)) return r;
  if (Cl.h < kHsF && G.h < kHsF) return r;
  // discharges in C's outward frame (normal, tangential)
  float cqn, cqt, gqn, gqt;
  if (side == 0) {
    cqn = Cl.qx; cqt = Cl.qy; gqn = G.qx; gqt = G.qy;
  } else if (side == 1) {
    cqn = Cl.qy; cqt = Cl.qx; gqn = G.qy; gqt = G.qx;
  } else if (side == 2) {
    cqn = -Cl.qx; cqt = -Cl.qy; gqn = -G.qx; gqt = -G.qy;
  } else {
    cqn = -Cl.qy; cqt = Cl.qx; gqn = -G.qy; gqt = G.qx;
  }
  f2 fh, fn, ft, sa, sb;
  // (every ghost has G.wl = G.z + G.h in C's frame, the free surface the
  // face core forms from the bed and the depth)
  face_core2<ORDER>(dup(Cl.h), dup(G.h), dup(G.z), dup(Cl.h), dup(0.f), dup(cqn), dup(cqt),
                    dup(G.h), dup(G.z), dup(gqn), dup(gqt), fh, fn, ft, sa, sb);
  r.sc = sa.x;
  if (side == 0) {  // C is the west side
    r.fh = fh.x; r.fx = fn.x; r.fy = ft.x;
  } else if (side == 1) {  // C is the south side
    r.fh = fh.x; r.fx = ft.x; r.fy = fn.x;
  } else if (side == 2) {  // C is the east side: the face's flux is minus C's outflow
    r.fh = -fh.x; r.fx = fn.x; r.fy = ft.x;
  } else {  // C is the north side
    r.fh = -fh.x; r.fx = -ft.x; r.fy = fn.x;
  }
  return r;
}

// ---------------------------------------------------------------------------
// Shared memory of a 64 x TY tile
// ---------------------------------------------------------------------------
constexpr int kPW = 64;             // tile width: 32 lanes x 2 cells
constexpr int kPSWF = kPW + 8;      // staged field row: cols -4 .. 67
constexpr int kPSWC = kPW + 32;     // staged code row: cols -16 .. 79

template <int TY>
struct PairSmem {
  static constexpr int SH = TY + 4;
  static constexpr int R = TY / kRowsNW;
  float f[4][SH * kPSWF];     // h, qx, qy, z
  float hmax[TY * kPW];
  uint8_t code[SH * kPSWC];
  alignas(8) unsigned long long bar;
  float xe[TY][4];            // face between cols 63 | 64: fh, fx, fy, sa
  float sxw[TY][4];           // x-slope of col -1: h, z, qx, qy
  double bc[HB_MAX_CLASSES][4];
  int bctype[HB_MAX_CLASSES];
  float manning[HB_MAX_ZONES];
  float ddatum[9];
  double red_d[2][kRowsNW];
  double red_s[kRowsNW];
  int red_i[kRowsNW];
  int last;
  int last2;
  unsigned rowmask;           // general tiles: bit i set if row i holds a valid cell
  static constexpr unsigned kTxBytes =
      (unsigned)(4 * SH * kPSWF * sizeof(float) + TY * kPW * sizeof(float) + SH * kPSWC);
};

template <int TY>
struct PairView {
  const PairSmem<TY> &s;
  __device__ __forceinline__ int fi(int i, int j) const { return (i + 2) * kPSWF + (j + 4); }
  __device__ __forceinline__ uint8_t code(int i, int j) const {
    return s.code[(i + 2) * kPSWC + (j + 16)];
  }
  // cells (i, j) and (i, j + 1), j even
  __device__ __forceinline__ Cel2 pair(int i, int j) const {
    const int k = fi(i, j);
    Cel2 c;
    c.h = *reinterpret_cast<const f2 *>(&s.f[0][k]);
    c.qx = *reinterpret_cast<const f2 *>(&s.f[1][k]);
    c.qy = *reinterpret_cast<const f2 *>(&s.f[2][k]);
    c.z = *reinterpret_cast<const f2 *>(&s.f[3][k]);
    return c;
  }
  // cells (i, j) and (i + 1, j): a vertical pair (tile-edge pre-pass)
  __device__ __forceinline__ Cel2 vpair(int i, int j) const {
    const int k = fi(i, j);
    Cel2 c;
    c.h = pk(s.f[0][k], s.f[0][k + kPSWF]);
    c.qx = pk(s.f[1][k], s.f[1][k + kPSWF]);
    c.qy = pk(s.f[2][k], s.f[2][k + kPSWF]);
    c.z = pk(s.f[3][k], s.f[3][k + kPSWF]);
    return c;
  }
  __device__ __forceinline__ float v(int fld, int i, int j) const { return s.f[fld][fi(i, j)]; }
};

// x-slopes of cell (i, j) (each field) from its west and east neighbours; an
// invalid neighbour is replaced by the cell itself
// (HC/flucCal_2ndOrder_jh_improved_Kernel.cu:416-428)
template <int TY, bool ALLV>
__device__ __forceinline__ void xslope1(const PairView<TY> &V, int i, int j, float &sh, float &sz,
                                        float &sqx, float &sqy) {
  bool vw = true, ve = true;
  if constexpr (!ALLV) {
    vw = is_valid(V.code(i, j - 1));
    ve = is_valid(V.code(i, j + 1));
  }
  const int k = V.fi(i, j);
  float c[4], w[4], e[4], o[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    c[q] = V.s.f[q][k];
    w[q] = vw ? V.s.f[q][k - 1] : c[q];
    e[q] = ve ? V.s.f[q][k + 1] : c[q];
    o[q] = slope1(c[q], w[q], e[q]);
  }
  sh = o[0];
  sqx = o[1];
  sqy = o[2];
  sz = o[3];
}

// y-slopes of the pair c (minus side = south row s, plus side = north row n)
template <bool ALLV>
__device__ __forceinline__ Slp2 yslope2(const Cel2 &c, const Cel2 &s, f2 vs, const Cel2 &n, f2 vn) {
  Cel2 m = s, p = n;
  if constexpr (!ALLV) {
    if (vs.x == 0.f) { m.h.x = c.h.x; m.qx.x = c.qx.x; m.qy.x = c.qy.x; m.z.x = c.z.x; }
    if (vs.y == 0.f) { m.h.y = c.h.y; m.qx.y = c.qx.y; m.qy.y = c.qy.y; m.z.y = c.z.y; }
    if (vn.x == 0.f) { p.h.x = c.h.x; p.qx.x = c.qx.x; p.qy.x = c.qy.x; p.z.x = c.z.x; }
    if (vn.y == 0.f) { p.h.y = c.h.y; p.qx.y = c.qx.y; p.qy.y = c.qy.y; p.z.y = c.z.y; }
  }
  Slp2 o;
  o.h = slope2(c.h, m.h, p.h);
  o.z = slope2(c.z, m.z, p.z);
  o.qx = slope2(c.qx, m.qx, p.qx);
  o.qy = slope2(c.qy, m.qy, p.qy);
  return o;
}

// Interior pair of faces, with the ghost and no-data cases of the general
// build fixed up per face: va / vb say whether side A / B of each face is a
// valid cell; ca / cb are their codes.  DIR 0: A is the west side, DIR 1 the
// south side.
template <int DIR, bool ALLV, int TY, int ORDER = 2>
__device__ __forceinline__ Fc2 face_pair(const PairSmem<TY> &s, const Cel2 &A, const Cel2 &B,
                                         const Slp2 &sA, const Slp2 &sB, uint8_t ca0,
                                         uint8_t ca1, uint8_t cb0, uint8_t cb1, float datum) {
  Fc2 o = face2<DIR, ORDER>(A, B, sA, sB);
  if constexpr (!ALLV) {
    const bool va0 = is_valid(ca0), va1 = is_valid(ca1), vb0 = is_valid(cb0), vb1 = is_valid(cb1);
    if (!(va0 && vb0) || !(va1 && vb1)) {
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const bool va = c ? va1 : va0, vb = c ? vb1 : vb0;
        if (va && vb) continue;
        Ghost1 gr{0.f, 0.f, 0.f, 0.f};
        float sa = 0.f, sb = 0.f;
        if (va) {
          const int cls = (c ? ca1 : ca0) >> 4;
          gr = ghost_face1<ORDER>(c ? A.h.y : A.h.x, c ? A.qx.y : A.qx.x, c ? A.qy.y : A.qy.x,
                                  c ? A.z.y : A.z.x, s.bctype[cls], s.bc[cls], datum,
                                  DIR == 0 ? 0 : 1);
          sa = gr.sc;
        } else if (vb) {
          const int cls = (c ? cb1 : cb0) >> 4;
          gr = ghost_face1<ORDER>(c ? B.h.y : B.h.x, c ? B.qx.y : B.qx.x, c ? B.qy.y : B.qy.x,
                                  c ? B.z.y : B.z.x, s.bctype[cls], s.bc[cls], datum,
                                  DIR == 0 ? 2 : 3);
          sb = gr.sc;
        }
        if (c) {
          o.fh.y = gr.fh; o.fx.y = gr.fx; o.fy.y = gr.fy; o.sa.y = sa; o.sb.y = sb;
        } else {
          o.fh.x = gr.fh; o.fx.x = gr.fx; o.fy.x = gr.fy; o.sa.x = sa; o.sb.x = sb;
        }
      }
    }
  }
  return o;
}

// ===========================================================================
// One tile of a step (FP32, scheme ORDER 2 or 1): stage it, evaluate its faces, update
// its cells, write its partial sums, and close its group / finalize its
// instance when it is the last.  PATH 0: a general tile (no-data cells, ghost
// faces or the cell-0 rule's cell in reach); PATH 1: an all-valid tile.
// Returns false when the tile's data did not arrive within the bounded wait
// (the instance's status says so; the caller leaves).
// ===========================================================================
// One tile: en = its TileEntry (en.tile < 0: ~tile of a general tile that
// holds no valid cell, which loads nothing and adds a zero partial to its
// group).
template <int TY, bool SOURCES, int PATH, int ORDER = 2>
__device__ __forceinline__ bool pair_tile(PairSmem<TY> &s, unsigned &phase, const TileEntry en,
                                          const hb_instance *__restrict__ insts,
                                          TilePartial *__restrict__ partials,
                                          TilePartial *__restrict__ gparts,
                                          unsigned *__restrict__ gcount, BcTable *__restrict__ bct,
                                          const CUtensorMap *__restrict__ maps) {
  constexpr bool kAllValid = PATH == 1;
  constexpr bool ALLV = kAllValid;
  const bool skip = !kAllValid && en.tile < 0;
  const int tile = en.tile < 0 ? ~en.tile : en.tile;
  using S = PairSmem<TY>;
  constexpr int R = S::R;
  const PairView<TY> V{s};
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int ii = en.inst;
  const hb_instance &in = insts[ii];
  hb_ctrl *ctrl = en.ctrl;
  if (__ldcg(&ctrl->halted)) return true;
  const int lt = tile - in.tile_begin;
  const int tyi = lt / in.tiles_x, txi = lt - tyi * in.tiles_x;
  const int y0 = tyi * TY, x0 = txi * kPW;
  // the control block changes between steps (a persistent launch reads it
  // again after every grid barrier): loads that bypass L1
  const int cur = __ldcg(&ctrl->cur);
  const double t = __ldcg(&ctrl->t);
  const float dt = (float)__ldcg(&ctrl->dt);
  const float dx = (float)in.dx;
  const float rain = (float)__ldcg(&ctrl->rain_rate);
  const bool first = (t == 0.0);
  const int P = in.pitch;
  const CUtensorMap *m = maps + (size_t)ii * kMapsPerInstance;

  if (tid == 0 && !skip) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&s.bar, S::kTxBytes);
    tma_load_2d(s.f[0], m + 0 + cur, x0, y0, &s.bar);
    tma_load_2d(s.f[1], m + 2 + cur, x0, y0, &s.bar);
    tma_load_2d(s.f[2], m + 4 + cur, x0, y0, &s.bar);
    tma_load_2d(s.f[3], m + 6, x0, y0, &s.bar);
    tma_load_2d(s.hmax, m + 7, x0 + HB_PAD_X, y0 + HB_PAD_Y, &s.bar);
    tma_load_2d(s.code, m + 8, x0, y0, &s.bar);
  }
  if (tid < HB_MAX_CLASSES) {
    if constexpr (!kAllValid) {
      s.bctype[tid] = in.bc_type[tid];
      for (int q = 0; q < 4; q++) s.bc[tid][q] = __ldcg(&bct[ii].v[tid][q]);
    }
  } else if (tid >= 64 && tid < 64 + HB_MAX_ZONES) {
    s.manning[tid - 64] = (float)in.manning[tid - 64];
  }
  const int bug_y = in.bug_y, bug_x = in.bug_x;
  float datum_tile = 0.f;
  if (in.datum && !skip) {
    const int by = y0 / HB_DATUM_BLOCK, bx = x0 / HB_DATUM_BLOCK;
    datum_tile = in.datum[by * in.datum_nx + bx];
    if (tid >= 32 && tid < 41) {
      const int q = tid - 32, dyb = q / 3 - 1, dxb = q % 3 - 1;
      const int yy = min(max(by + dyb, 0), in.datum_ny - 1);
      const int xx = min(max(bx + dxb, 0), in.datum_nx - 1);
      s.ddatum[q] = in.datum[yy * in.datum_nx + xx] - datum_tile;
    }
  }
  if (!skip) {
    const bool arrived = mbar_wait(&s.bar, phase, 4000000000LL);
    if (__syncthreads_or(!arrived)) {
      if (tid == 0) atomicOr(&ctrl->status, 2);
      mbar_wait(&s.bar, phase, 4000000000LL);
      return false;
    }
    phase ^= 1u;
  }
  if constexpr (!ALLV) {
    // rows of the tile that hold a valid cell (lane i: row i, 16 words of 4
    // codes; a code is valid unless its class nibble is the no-data class)
    if (w == 0) {
      bool rv = false;
      if (!skip && lane < TY) {
        const uint32_t *row = reinterpret_cast<const uint32_t *>(&s.code[(lane + 2) * kPSWC + 16]);
#pragma unroll
        for (int q = 0; q < kPW / 4; ++q)
          rv = rv || (row[q] & 0xF0F0F0F0u) != 0xF0F0F0F0u;
      }
      const unsigned m = __ballot_sync(0xffffffffu, rv);
      if (lane == 0) s.rowmask = m;
    }
  }
  if (in.datum && !skip) {
    __syncthreads();  // ddatum visible
    const int by0 = (y0 / HB_DATUM_BLOCK) * HB_DATUM_BLOCK;
    const int bx0 = (x0 / HB_DATUM_BLOCK) * HB_DATUM_BLOCK;
    const DatumHalo dh = datum_halo(y0, x0, by0, bx0, TY, kPW, kPSWF, HB_DATUM_BLOCK);
    const int NH = dh.count();
    for (int q = tid; q < NH; q += kRowsNT) {
      int i, j;
      datum_halo_cell(dh, q, TY, kPW, kPSWF, i, j);
      const int ry = y0 + i, rx = x0 + j;
      const int dyb = ry < by0 ? 0 : (ry >= by0 + HB_DATUM_BLOCK ? 2 : 1);
      const int dxb = rx < bx0 ? 0 : (rx >= bx0 + HB_DATUM_BLOCK ? 2 : 1);
      if (dyb != 1 || dxb != 1) s.f[3][V.fi(i, j)] += s.ddatum[dyb * 3 + dxb];
    }
  }
  __syncthreads();

  // --- tile edges: warp 0 the faces between columns 63 | 64 (east faces of
  // lane 31's second cell), two rows per lane; warp 1 the x-slopes of
  // column -1 (west neighbour of lane 0's first cell)
  if (skip) {
  } else if (w == 0) {
    for (int i = 2 * lane; i < TY; i += 64) {
      float a[4], b[4];  // slopes of col 63 / col 64 for rows i, i + 1 (h, z, qx, qy)
      float a1[4], b1[4];
      xslope1<TY, ALLV>(V, i, 63, a[0], a[1], a[2], a[3]);
      xslope1<TY, ALLV>(V, i + 1, 63, a1[0], a1[1], a1[2], a1[3]);
      xslope1<TY, ALLV>(V, i, 64, b[0], b[1], b[2], b[3]);
      xslope1<TY, ALLV>(V, i + 1, 64, b1[0], b1[1], b1[2], b1[3]);
      const Slp2 sA{pk(a[0], a1[0]), pk(a[1], a1[1]), pk(a[2], a1[2]), pk(a[3], a1[3])};
      const Slp2 sB{pk(b[0], b1[0]), pk(b[1], b1[1]), pk(b[2], b1[2]), pk(b[3], b1[3])};
      const Fc2 f = face_pair<0, ALLV, TY, ORDER>(s, V.vpair(i, 63), V.vpair(i, 64), sA, sB,
                                       V.code(i, 63), V.code(i + 1, 63), V.code(i, 64),
                                       V.code(i + 1, 64), datum_tile);
      s.xe[i][0] = f.fh.x; s.xe[i][1] = f.fx.x; s.xe[i][2] = f.fy.x; s.xe[i][3] = f.sa.x;
      s.xe[i + 1][0] = f.fh.y; s.xe[i + 1][1] = f.fx.y; s.xe[i + 1][2] = f.fy.y;
      s.xe[i + 1][3] = f.sa.y;
    }
  } else if (w == 1) {
    for (int i = lane; i < TY; i += 32) {
      float sh, sz, sqx, sqy;
      xslope1<TY, ALLV>(V, i, -1, sh, sz, sqx, sqy);
      s.sxw[i][1] = sz;
      if constexpr (ORDER == 2) {  // the 1st-order faces read only the bed's slope
        s.sxw[i][0] = sh;
        s.sxw[i][2] = sqx;
        s.sxw[i][3] = sqy;
      }
    }
  }

  // rows walked by this warp: all-valid tiles R rows each; general tiles
  // share the rows from the first to the last one that holds a valid cell
  // evenly among the warps (a tile over the catchment's edge with a few live
  // rows then takes a few rows' time), none when the tile is empty
  int r0 = w * R, r_end = r0 + R;
  if constexpr (!ALLV) {
    const unsigned m = s.rowmask;  // written before the barrier above
    const int lo = m ? __ffs(m) - 1 : 0, hi = m ? 32 - __clz(m) : 0;
    r0 = lo + (w * (hi - lo)) / kRowsNW;
    r_end = lo + ((w + 1) * (hi - lo)) / kRowsNW;
  }
  const int j0 = 2 * lane;  // this lane's first column
  const int rx0 = x0 + j0;
  f2 vol2 = dup(0.f);
  float smax_t = 0.f;
  double outf = 0.0;
  int any_dry = 0;
  {
    // validity of a pair as two floats (1 valid, 0 not); all-valid: 1
    auto vpair = [&](int i) -> f2 {
      if constexpr (ALLV) {
        (void)i;
        return dup(1.f);
      } else {
        return pk(is_valid(V.code(i, j0)) ? 1.f : 0.f, is_valid(V.code(i, j0 + 1)) ? 1.f : 0.f);
      }
    };
    // --- column window of the pair: row r0 and its y-slopes, the face
    // between rows r0-1 and r0, the depths of row r0-1
    Cel2 C = V.pair(r0, j0);
    f2 vC = vpair(r0), vN = vpair(r0 - 1);
    f2 Nh;
    Slp2 syC;
    Fc2 nf;
    {
      const Cel2 N = V.pair(r0 - 1, j0), NN = V.pair(r0 - 2, j0), S1 = V.pair(r0 + 1, j0);
      const Slp2 syN = yslope2<ALLV>(N, C, vC, NN, vpair(r0 - 2));
      syC = yslope2<ALLV>(C, S1, vpair(r0 + 1), N, vN);
      // face between rows r0-1 (north, B) and r0 (south, A)
      nf = face_pair<1, ALLV, TY, ORDER>(s, C, N, syC, syN, V.code(r0, j0), V.code(r0, j0 + 1),
                              V.code(r0 - 1, j0), V.code(r0 - 1, j0 + 1), datum_tile);
      Nh = N.h;
    }
    __syncthreads();  // tile-edge faces and slopes ready
    float *hout = (float *)in.h[1 - cur];
    float *qxout = (float *)in.qx[1 - cur];
    float *qyout = (float *)in.qy[1 - cur];
    float *hmaxg = (float *)in.h_max;
    const bool infil = SOURCES && in.cum != nullptr;
    const bool stations = SOURCES && in.rain_station != nullptr;
    const bool fwd_tile = (y0 < HB_PAD_Y && in.halo_up[0] != nullptr) ||
                          (y0 + TY > in.rows - HB_PAD_Y && in.halo_down[0] != nullptr);
    const f2 r2 = dup(dt / dx);
    const float rdt = rain * dt;
    const float dtg = dt * kGF;

#pragma unroll 1
    for (int i = r0; i < r_end; ++i) {
      // --- x-direction: neighbours W (col 2j-1) and E (col 2j+2)
      const int kc = V.fi(i, j0);
      float Wv[4], Ev[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        Wv[q] = s.f[q][kc - 1];
        Ev[q] = s.f[q][kc + 2];
      }
      uint8_t kW = 0, kE = 0;
      const uint8_t kA = V.code(i, j0), kB = V.code(i, j0 + 1);
      bool vWb = true, vAb = true, vBb = true, vEb = true;
      if constexpr (!ALLV) {
        kW = V.code(i, j0 - 1);
        kE = V.code(i, j0 + 2);
        vWb = is_valid(kW);
        vAb = is_valid(kA);
        vBb = is_valid(kB);
        vEb = is_valid(kE);
      }
      // x-slopes of cells a = 2j and b = 2j+1 (fields h, qx, qy, z)
      const float cA[4] = {C.h.x, C.qx.x, C.qy.x, C.z.x};
      const float cB[4] = {C.h.y, C.qx.y, C.qy.y, C.z.y};
      float sxa[4], sxb[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        sxa[q] = slope1(cA[q], vWb ? Wv[q] : cA[q], vBb ? cB[q] : cA[q]);
        sxb[q] = slope1(cB[q], vAb ? cA[q] : cB[q], vEb ? Ev[q] : cB[q]);
      }
      // slope of col 2j-1 from the west lane (lane 0: the pre-pass); the
      // 1st-order faces read only the bed's
      float sw[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (ORDER == 2 || q == 3) sw[q] = __shfl_up_sync(0xffffffffu, sxb[q], 1);
      if (lane == 0) {
        sw[3] = s.sxw[i][1];
        if constexpr (ORDER == 2) {
          sw[0] = s.sxw[i][0];
          sw[1] = s.sxw[i][2];
          sw[2] = s.sxw[i][3];
        }
      }
      // --- west faces of a and b: (2j-1 | 2j) and (2j | 2j+1)
      f2 Px_h, Px_x, Px_y;  // x-direction flux differences (west - east) of the pair
      f2 wfh;               // west-face mass flux (outflow of boundary faces)
      f2 efh;               // east-face mass flux
      {
        const Cel2 Aw{pk(Wv[0], C.h.x), pk(Wv[1], C.qx.x), pk(Wv[2], C.qy.x), pk(Wv[3], C.z.x)};
        const Slp2 sAw{pk(sw[0], sxa[0]), pk(sw[3], sxa[3]), pk(sw[1], sxa[1]), pk(sw[2], sxa[2])};
        const Slp2 sBw{pk(sxa[0], sxb[0]), pk(sxa[3], sxb[3]), pk(sxa[1], sxb[1]), pk(sxa[2], sxb[2])};
        const Fc2 wf = face_pair<0, ALLV, TY, ORDER>(s, Aw, C, sAw, sBw, kW, kA, kA, kB,
                                                     datum_tile);
        // east faces: a's is the lane's second west face; b's comes from lane j+1
        float e_h = __shfl_down_sync(0xffffffffu, wf.fh.x, 1);
        float e_x = __shfl_down_sync(0xffffffffu, wf.fx.x, 1);
        float e_y = __shfl_down_sync(0xffffffffu, wf.fy.x, 1);
        float e_a = __shfl_down_sync(0xffffffffu, wf.sa.x, 1);
        if (lane == 31) {
          e_h = s.xe[i][0];
          e_x = s.xe[i][1];
          e_y = s.xe[i][2];
          e_a = s.xe[i][3];
        }
        const f2 ef_h = pk(wf.fh.y, e_h), ef_x = pk(wf.fx.y, e_x), ef_y = pk(wf.fy.y, e_y),
                 ef_a = pk(wf.sa.y, e_a);
        Px_h = sub2(wf.fh, ef_h);
        Px_x = add2(sub2(sub2(wf.fx, ef_x), ef_a), wf.sb);
        Px_y = sub2(wf.fy, ef_y);
        wfh = wf.fh;
        efh = ef_h;
      }
      // --- the row below, its y-slopes, and the south faces: rows i+1 (A) | i (B)
      const Cel2 Sx = V.pair(i + 1, j0);
      const f2 vS = vpair(i + 1);
      Fc2 sf;
      Slp2 syS;
      {
        const Cel2 SS = V.pair(i + 2, j0);
        syS = yslope2<ALLV>(Sx, SS, vpair(i + 2), C, vC);
        uint8_t kSa = 0, kSb = 0;
        if constexpr (!ALLV) {
          kSa = V.code(i + 1, j0);
          kSb = V.code(i + 1, j0 + 1);
        }
        sf = face_pair<1, ALLV, TY, ORDER>(s, Sx, C, syS, syC, kSa, kSb, kA, kB, datum_tile);
      }

      // --- cell updates
      const int ry = y0 + i;
      // fluxMask activity (HC/fluxMaskGenerator_Kernel.cu:19-42)
      bool act0 = first || C.h.x > kHsF, act1 = first || C.h.y > kHsF;
      if (!(act0 && act1)) {
        if constexpr (ALLV) {
          act0 = act0 || C.h.y > kHsF || Nh.x > kHsF || Wv[0] > kHsF || Sx.h.x > kHsF;
          act1 = act1 || Ev[0] > kHsF || Nh.y > kHsF || C.h.x > kHsF || Sx.h.y > kHsF;
        } else {
          const int ra = rx0, rb = rx0 + 1;
          auto nb = [&](bool v, int yy, int xx, float hh) {
            return v && !(yy == bug_y && xx == bug_x) && hh > kHsF;
          };
          act0 = act0 || nb(vBb, ry, ra + 1, C.h.y) || nb(vN.x != 0.f, ry - 1, ra, Nh.x) ||
                 nb(vWb, ry, ra - 1, Wv[0]) || nb(vS.x != 0.f, ry + 1, ra, Sx.h.x);
          act1 = act1 || nb(vEb, ry, rb + 1, Ev[0]) || nb(vN.y != 0.f, ry - 1, rb, Nh.y) ||
                 nb(vAb, ry, rb - 1, C.h.x) || nb(vS.y != 0.f, ry + 1, rb, Sx.h.y);
        }
      }
      f2 hu = mul2(add2(Px_h, sub2(sf.fh, nf.fh)), r2);
      f2 qxu = mul2(add2(Px_x, sub2(sf.fx, nf.fx)), r2);
      f2 qyu = mul2(add2(Px_y, add2(sub2(sub2(sf.fy, nf.fy), nf.sa), sf.sb)), r2);
      if (!act0) hu.x = qxu.x = qyu.x = 0.f;
      if (!act1) hu.y = qxu.y = qyu.y = 0.f;
      if constexpr (!ALLV) {
        // outflow through boundary faces of active valid cells
        const bool bE0 = !vBb, bW0 = !vWb, bN0 = vN.x == 0.f, bS0 = vS.x == 0.f;
        const bool bE1 = !vEb, bW1 = !vAb, bN1 = vN.y == 0.f, bS1 = vS.y == 0.f;
        if (vAb && act0 && (bE0 | bW0 | bN0 | bS0)) {
          double o = 0.0;
          if (bE0) o += (double)efh.x;
          if (bN0) o += (double)nf.fh.x;
          if (bW0) o -= (double)wfh.x;
          if (bS0) o -= (double)sf.fh.x;
          outf += o;
        }
        if (vBb && act1 && (bE1 | bW1 | bN1 | bS1)) {
          double o = 0.0;
          if (bE1) o += (double)efh.y;
          if (bN1) o += (double)nf.fh.y;
          if (bW1) o -= (double)wfh.y;
          if (bS1) o -= (double)sf.fh.y;
          outf += o;
        }
      }
      // rain (HP/SWE_CUDA.py:549 / HC/stationPrecipitation_Kernel.cu:27)
      const size_t go = (size_t)(ry + HB_PAD_Y) * P + (rx0 + HB_PAD_X);
      if (stations) {
        hu.x += (float)__ldcg(&in.station_rate[in.rain_station[go]]) * dt;
        hu.y += (float)__ldcg(&in.station_rate[in.rain_station[go + 1]]) * dt;
      } else {
        hu = add2(hu, dup(rdt));
      }
      if (infil) {
        // Green-Ampt infiltration on the active cells, after rain
        // (HC/infiltrationCUDA_Kernel.cu:20-46; order HP/CatchFlood_main.py:164-170)
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const bool act = c ? act1 : act0;
          const bool vc = c ? vBb : vAb;
          if (!(act && vc)) continue;
          const uint8_t kc_ = c ? kB : kA;
          const float hc = c ? C.h.y : C.h.x;
          float *cum = (float *)in.cum + go + c;
          const int zc = kc_ & 15;
          const float K = (float)in.ks[zc], psi = (float)in.psi[zc], dth = (float)in.dtheta[zc];
          const float F0 = *cum;
          const float a = F0 + dt * K;
          const float F1 = 0.5f * (a + sqrtf(a * a + 4.f * dt * K * (psi + hc) * dth));
          const float dF = fminf(hc, F1 - F0);
          *cum = F0 + dF;
          if (c) hu.y -= dF; else hu.x -= dF;
        }
      }
      // implicit friction + update (HC/friction_implicit_andUpdate_jh_Kernel.cu:22-146)
      const f2 h2 = add2(C.h, hu);
      f2 qx2 = add2(C.qx, qxu), qy2 = add2(C.qy, qyu);
      f2 sgh = dup(0.f), ih = dup(0.f);
      const f2 nman = pk(s.manning[kA & 15], s.manning[kB & 15]);
      {
        const f2 gh = mul2(dup(kGF), h2);
        sgh = pk(sqrta(gh.x), sqrta(gh.y));
        ih = pk(rcpa(h2.x), rcpa(h2.y));
        const f2 qq = fma2(qx2, qx2, mul2(qy2, qy2));
        const f2 qn = pk(sqrta(qq.x), sqrta(qq.y));
        const f2 cb = pk(ex2a(lg2a(h2.x) * (-1.f / 3.f)), ex2a(lg2a(h2.y) * (-1.f / 3.f)));
        const f2 a = mul2(mul2(mul2(mul2(mul2(dup(dtg), nman), nman), cb), ih), ih);
        const f2 sq = fma2(mul2(dup(4.f), a), qn, dup(1.f));
        const f2 den = add2(dup(1.f), pk(sqrta(sq.x), sqrta(sq.y)));
        const f2 fct = pk(2.f * rcpa(den.x), 2.f * rcpa(den.y));
        const f2 lim = mul2(mul2(dup(5.f), h2), sgh);
        const f2 tx = mul2(qx2, fct), ty = mul2(qy2, fct);
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const float hh = c ? h2.y : h2.x;
          float &qx = c ? qx2.y : qx2.x;
          float &qy = c ? qy2.y : qy2.x;
          // The limiter as selects: a dry cell stops (q = 0), a cell without
          // Manning friction keeps q, a wet one takes the implicit value,
          // over-corrected (2 temp - q, clipped at a sign change) where
          // |temp| passes 5 h sqrt(gh), and q itself is kept at |q| <= 1e-10.
          // The values a dry or friction-free cell computes here (inf or NaN
          // at h = 0) are never selected. Same results as the branching form,
          // without the divergent branches around the two components.
          const float l = c ? lim.y : lim.x;
          auto limit = [&](float q, float temp) {
            const float q2 = 2.f * temp - q;
            const float over = (q2 * temp <= 0.f) ? 0.f : q2;
            const float t = fabsf(temp) > l ? over : temp;
            return fabsf(q) > 1.0e-10f ? t : q;
          };
          const bool fr = (c ? nman.y : nman.x) > 0.f, wet = !(hh < kHsF);
          const float nqx = limit(qx, c ? tx.y : tx.x), nqy = limit(qy, c ? ty.y : ty.x);
          // (sgh, ih of a dry cell: the CFL speed below skips dry cells)
          qx = wet ? (fr ? nqx : qx) : 0.f;
          qy = wet ? (fr ? nqy : qy) : 0.f;
        }
      }
      // stores: both cells valid (every all-valid tile), else per cell
      const f2 hm_old = *reinterpret_cast<const f2 *>(&s.hmax[i * kPW + j0]);
      const f2 hm = pk(fmaxf(h2.x, hm_old.x), fmaxf(h2.y, hm_old.y));
      if (vAb && vBb) {
        *reinterpret_cast<f2 *>(hout + go) = h2;
        *reinterpret_cast<f2 *>(qxout + go) = qx2;
        *reinterpret_cast<f2 *>(qyout + go) = qy2;
        *reinterpret_cast<f2 *>(hmaxg + go) = hm;
      } else {
        if (vAb) {
          hout[go] = h2.x; qxout[go] = qx2.x; qyout[go] = qy2.x; hmaxg[go] = hm.x;
        }
        if (vBb) {
          hout[go + 1] = h2.y; qxout[go + 1] = qx2.y; qyout[go + 1] = qy2.y; hmaxg[go + 1] = hm.y;
        }
      }
      if (fwd_tile) {
        const int ob = 1 - cur;
        auto fwd = [&](void *const *dst, int row) {
          const size_t gh = (size_t)row * P + (rx0 + HB_PAD_X);
          if (vAb) {
            ((float *)dst[ob])[gh] = h2.x;
            ((float *)dst[2 + ob])[gh] = qx2.x;
            ((float *)dst[4 + ob])[gh] = qy2.x;
          }
          if (vBb) {
            ((float *)dst[ob])[gh + 1] = h2.y;
            ((float *)dst[2 + ob])[gh + 1] = qx2.y;
            ((float *)dst[4 + ob])[gh + 1] = qy2.y;
          }
        };
        if (ry < HB_PAD_Y && in.halo_up[0] != nullptr)
          fwd(in.halo_up, in.halo_up_rows + HB_PAD_Y + ry);
        if (ry >= in.rows - HB_PAD_Y && in.halo_down[0] != nullptr)
          fwd(in.halo_down, ry - in.rows + HB_PAD_Y);
        // the neighbour may be a peer GPU: order these stores system-wide
        // before this tile's partial, its group count and the host's next
        // collective
        __threadfence_system();
      }
      // CFL speed (HC/timeControl_Kernel.cu:186-189), volume
      const f2 sp = fma2(pk(fmaxf(fabsf(qx2.x), fabsf(qy2.x)), fmaxf(fabsf(qx2.y), fabsf(qy2.y))),
                         ih, sgh);
      if (vAb) {
        if (h2.x > kHsF) smax_t = fmaxf(smax_t, sp.x); else any_dry = 1;
      }
      if (vBb) {
        if (h2.y > kHsF) smax_t = fmaxf(smax_t, sp.y); else any_dry = 1;
      }
      vol2 = add2(vol2, pk(vAb ? h2.x : 0.f, vBb ? h2.y : 0.f));

      // slide the column window down one row
      nf = sf;
      Nh = C.h;
      vN = vC;
      C = Sx;
      vC = vS;
      syC = syS;
    }
  }

  // --- tile partials and the instance's last-tile finalize
  double vol = warp_sum((double)vol2.x + (double)vol2.y);
  if constexpr (!kAllValid) outf = warp_sum(outf);
  const double smax = (double)warp_max(smax_t);
  any_dry = __any_sync(0xffffffffu, any_dry);
  if (lane == 0) {
    s.red_d[0][w] = vol;
    s.red_d[1][w] = outf;
    s.red_s[w] = smax;
    s.red_i[w] = any_dry;
  }
  __syncthreads();
  const int n_inst_tiles = in.tiles_x * in.tiles_y;
  const int grp = lt / kGroupTiles;
  const int gsize = min(kGroupTiles, n_inst_tiles - grp * kGroupTiles);
  const int gbase = in.tile_begin / kGroupTiles + ii;
  if (tid == 0) {
    TilePartial p;
    p.volume = p.outflow = p.smax = 0.0;
    p.any_dry = 0;
    p.pad = 0;
    for (int q = 0; q < kRowsNW; q++) {
      p.volume += s.red_d[0][q];
      p.outflow += s.red_d[1][q];
      p.smax = fmax(p.smax, s.red_s[q]);
      p.any_dry |= s.red_i[q];
    }
    partials[tile] = p;
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> done(gcount[gbase + grp]);
    s.last = (done.fetch_add(1u, cuda::memory_order_acq_rel) == (unsigned)(gsize - 1));
  }
  __syncthreads();
  if (s.last)
    close_group<float, kRowsNT>(in, ii, partials + in.tile_begin + grp * kGroupTiles, gsize,
                                gparts, gcount, gbase + grp, gbase,
                                (n_inst_tiles + kGroupTiles - 1) / kGroupTiles, bct, s.red_d,
                                s.red_s, s.red_i, &s.last2);
  __syncthreads();
  return true;
}

// The step kernel: one launch per step and build, one CTA per tile by
// default (a positive grid loops over the build's tiles).  Tile k of the
// launch is list[k] before gap_at and list[k + gap_len] from there on (the
// general build skips the all-valid entries between its two parts).
template <int TY, int MINB, bool SOURCES, int PATH, int ORDER = 2>
__global__ void __launch_bounds__(kRowsNT, MINB)
pairs_step_kernel(const hb_instance *__restrict__ insts, const TileEntry *__restrict__ list,
                  const int n_list, const int gap_at, const int gap_len,
                  TilePartial *__restrict__ partials,
                  TilePartial *__restrict__ gparts,
                  unsigned *__restrict__ gcount, BcTable *__restrict__ bct,
                  const CUtensorMap *__restrict__ maps) {
  using S = PairSmem<TY>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);
  if (threadIdx.x == 0) {
    mbar_init(&s.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned phase = 0;
  for (int k = blockIdx.x; k < n_list; k += gridDim.x)
    if (!pair_tile<TY, SOURCES, PATH, ORDER>(s, phase, list[k < gap_at ? k : k + gap_len], insts,
                                             partials, gparts, gcount, bct, maps))
      return;
}

// ===========================================================================
// The persistent step: every instance of a batch advanced by nsteps steps in
// ONE cooperative launch of resident CTAs.  Per step, CTAs take tiles from a
// global counter in the prepared order (general tiles with a valid cell
// first, the tiles without one last), each tile runs
// exactly as in the per-step kernel (its instance's last tile finalizes the
// clock), and a grid barrier ends the step.  The barrier wait is bounded by
// `budget` clock cycles: a CTA that gives up sets the give-up flag and bit 8
// of every instance's status and leaves, and every other CTA leaves at its
// next wait when it sees the flag; nothing waits without bound.
// sync[0] counts tile fetches (every CTA makes exactly one failed fetch per
// step, so step k's fetches start at k * (n_tiles + gridDim.x)), sync[1] the
// barrier arrivals, sync[2] is the give-up flag; the host zeroes them before
// every launch.
// ===========================================================================
constexpr int kPersistMinBlocks = 4;

// A general tile of the persistent step, kept out of line so that the
// all-valid path inlined in the kernel gets the register allocation it gets in
// its own build (the general path's ghost faces would otherwise cost it spills).
template <int TY, bool SOURCES, int ORDER = 2>
__device__ __noinline__ bool pair_tile_general(PairSmem<TY> &s, unsigned &phase,
                                               const TileEntry en,
                                               const hb_instance *__restrict__ insts,
                                               TilePartial *__restrict__ partials,
                                               TilePartial *__restrict__ gparts,
                                               unsigned *__restrict__ gcount,
                                               BcTable *__restrict__ bct,
                                               const CUtensorMap *__restrict__ maps) {
  return pair_tile<TY, SOURCES, 0, ORDER>(s, phase, en, insts, partials, gparts, gcount, bct,
                                          maps);
}

// The step as ONE launch of one CTA per tile over the whole list: general
// tiles with a valid cell [0, n_live), all-valid tiles [n_live, n_valid_end),
// then the general tiles without a valid cell, which only add a zero partial
// and so take the slots the last wave leaves idle.  Every CTA has the all-valid build's
// register cap (4 CTAs per SM), so the two kinds share an SM's slots evenly;
// with the two builds as separate launches a general CTA (its own build needs
// ~160 registers) took the room of two all-valid ones while it ran, and the
// second launch started its tiles late.  A general tile runs the out-of-line
// general path and returns, so the all-valid path holds no values across a
// call and keeps the allocation of its own build.  Same results bit for bit
// as the two launches.
template <int TY, bool SOURCES, int ORDER>
__global__ void __launch_bounds__(kRowsNT, 4)
pairs_mixed_kernel(const hb_instance *__restrict__ insts, const TileEntry *__restrict__ list,
                   const int n_live, const int n_valid_end, const int n_list,
                   TilePartial *__restrict__ partials,
                   TilePartial *__restrict__ gparts, unsigned *__restrict__ gcount,
                   BcTable *__restrict__ bct, const CUtensorMap *__restrict__ maps) {
  using S = PairSmem<TY>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);
  if (threadIdx.x == 0) {
    mbar_init(&s.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned phase = 0;
  const int k = blockIdx.x;
  if (k < n_live || (k >= n_valid_end && k < n_list)) {
    pair_tile_general<TY, SOURCES, ORDER>(s, phase, list[k], insts, partials, gparts, gcount,
                                          bct, maps);
    return;
  }
  if (k < n_valid_end)
    pair_tile<TY, SOURCES, 1, ORDER>(s, phase, list[k], insts, partials, gparts, gcount, bct,
                                     maps);
}

template <int TY, bool SOURCES>
__global__ void __launch_bounds__(kRowsNT, kPersistMinBlocks)
pairs_persistent_kernel(const hb_instance *__restrict__ insts,
                        const TileEntry *__restrict__ entries,
                        const int32_t *__restrict__ counts, const uint8_t *__restrict__ allvalid,
                        TilePartial *__restrict__ partials, TilePartial *__restrict__ gparts,
                        unsigned *__restrict__ gcount, BcTable *__restrict__ bct,
                        const CUtensorMap *__restrict__ maps, int n_instances, int nsteps,
                        unsigned long long *__restrict__ sync, long long budget) {
  using S = PairSmem<TY>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);
  __shared__ unsigned long long s_tile;
  __shared__ int s_stop;
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&s.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned phase = 0;
  const unsigned long long n = (unsigned long long)(counts[0] + counts[1]);
  const unsigned long long G = gridDim.x;
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> fetches(sync[0]);
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> arrivals(sync[1]);
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> gave_up(sync[2]);
  for (int step = 0; step < nsteps; ++step) {
    const unsigned long long base = (unsigned long long)step * (n + G);
    for (;;) {
      if (tid == 0) s_tile = fetches.fetch_add(1ull, cuda::memory_order_relaxed) - base;
      __syncthreads();
      const unsigned long long k = s_tile;
      __syncthreads();
      if (k >= n) break;
      const TileEntry en = entries[k];
      const bool ok = en.tile >= 0 && allvalid[en.tile] == 1
                          ? pair_tile<TY, SOURCES, 1>(s, phase, en, insts, partials, gparts,
                                                      gcount, bct, maps)
                          : pair_tile_general<TY, SOURCES>(s, phase, en, insts, partials, gparts,
                                                           gcount, bct, maps);
      if (!ok) {
        if (tid == 0) gave_up.fetch_or(1ull, cuda::memory_order_relaxed);
        return;
      }
    }
    // --- grid barrier: this step's state stores (generic proxy) before the
    // next step's tile loads (TMA, async proxy) on any SM
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      arrivals.fetch_add(1ull, cuda::memory_order_release);
      const unsigned long long target = (unsigned long long)(step + 1) * G;
      const long long t0 = clock64();
      int stop = 0;
      while (arrivals.load(cuda::memory_order_acquire) < target) {
        if (gave_up.load(cuda::memory_order_relaxed)) {
          stop = 1;
          break;
        }
        if (clock64() - t0 > budget) {
          stop = 2;
          break;
        }
        __nanosleep(64);
      }
      // the last block to arrive skips the wait: it stops too if any block
      // gave up, so that no block carries on alone
      if (!stop && gave_up.load(cuda::memory_order_relaxed)) stop = 1;
      if (stop == 2) {
        gave_up.fetch_or(1ull, cuda::memory_order_relaxed);
        for (int i = 0; i < n_instances; i++) atomicOr(&insts[i].ctrl->status, 8);
      }
      asm volatile("fence.proxy.async.global;" ::: "memory");
      s_stop = stop;
    }
    __syncthreads();
    if (s_stop) return;
  }
}
