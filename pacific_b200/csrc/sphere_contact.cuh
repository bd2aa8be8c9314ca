// sphere_contact.cuh -- analytic closest points of sphere-sphere and
// sphere-box pairs, in double precision with every operation rounded
// separately so that contact decisions (overlap distance < 0) and ContactError
// tests equal the reference's bit for bit.
//
//   ClosestPointSPHERESPHERE : Geometry/src/RigidBodyWithCrust.cpp:596-639
//   ClosestPointSPHEREBOX    : Geometry/src/RigidBodyWithCrust.cpp:647-721
//   Box::IntersectionPointSPHERE + corner / edge helpers : Geometry/src/Box.cpp:466-768
#pragma once

#include "common.cuh"

namespace gg {

// PointContact (Geometry/include/PointContact.hh:119-131); no contact is
// overlap = 1e20 (PointNoContact, PointContact.hh:131)
struct ContactGeom {
  D3 point;
  D3 overlap_vector;
  double overlap;
  int status;  // 0 ok, 1 contact error (overlap >= crust sum or centre inside box)
};

GG_HD ContactGeom no_contact() {
  ContactGeom c;
  c.point = d3(0, 0, 0);
  c.overlap_vector = d3(0, 0, 0);
  c.overlap = 1.e20;
  c.status = 0;
  return c;
}

// Overlap distance of two spheres; the contact decision is overlap <= 0.
GG_HD double sphere_sphere_overlap(D3 a, double ra, D3 b, double rb, D3* ab, double* nab) {
  *ab = xsub3(b, a);
  *nab = xnorm(*ab);
  return xsub(*nab, xadd(ra, rb));
}

// Contact features once overlap <= 0 is known (RigidBodyWithCrust.cpp:613-638).
GG_HD ContactGeom sphere_sphere_features(D3 a, double ra, D3 ab, double nab, double dist, double crust_sum) {
  ContactGeom c;
  c.status = (-dist >= crust_sum) ? 1 : 0;
  // contact = A + (rA + dist/2) * AB / |AB|  (scale first, then divide)
  c.point = xadd3(a, xdivs(xscale(ab, xadd(ra, xmul(0.5, dist))), nab));
  // overlap_vector = dist * (AB / |AB|)
  c.overlap_vector = xscale(xdivs(ab, nab), dist);
  c.overlap = dist;
  return c;
}

// Box corner k in the order of Box::setCornersFaces (Box.cpp:92-111)
GG_HD D3 box_corner(D3 e, int k) {
  const bool px = (k == 1 || k == 2 || k == 5 || k == 6);
  const bool py = (k >= 4);
  const bool pz = (k == 2 || k == 3 || k == 6 || k == 7);
  return d3(px ? e.x : -e.x, py ? e.y : -e.y, pz ? e.z : -e.z);
}

// Box::ContactCornerSPHERE / ContactEdgeSPHERE (Box.cpp:724-768).  dir < 0
// selects the corner case, otherwise the edge parallel to axis dir.
GG_HD D3 box_feature_sphere(D3 e, D3 c, double r, int k, int dir, double* ov) {
  D3 cor = box_corner(e, k);
  D3 proj = c;
  if (dir == 0) proj.x = cor.x;
  if (dir == 1) proj.y = cor.y;
  if (dir == 2) proj.z = cor.z;
  D3 d = xsub3(proj, cor);
  double nd = xnorm(d);
  D3 cp = d3(0, 0, 0);
  if (nd < r) {
    *ov = xsub(nd, r);
    cp = xsub3(c, xscale(d, xadd(1., xdiv(xmul(0.5, *ov), nd))));
  }
  return cp;
}

// Box::IntersectionPointSPHERE in the box frame (Box.cpp:466-718).  Returns
// the contact point; *ov = overlap (< 0 on contact, 1 otherwise); *inside = 1
// when the sphere centre lies inside the box (a ContactError in the reference).
GG_HD D3 box_sphere_local(D3 e, D3 c, double r, double* ov, int* inside) {
  D3 cp = d3(0, 0, 0);
  double gx = c.x, gy = c.y, gz = c.z, nd;
  *ov = 1.;
  *inside = 0;
  if (gx > e.x) {
    if (gy > e.y) {
      if (gz > e.z) cp = box_feature_sphere(e, c, r, 6, -1, ov);
      else if (gz < -e.z) cp = box_feature_sphere(e, c, r, 5, -1, ov);
      else cp = box_feature_sphere(e, c, r, 5, 2, ov);
    } else if (gy < -e.y) {
      if (gz > e.z) cp = box_feature_sphere(e, c, r, 2, -1, ov);
      else if (gz < -e.z) cp = box_feature_sphere(e, c, r, 1, -1, ov);
      else cp = box_feature_sphere(e, c, r, 1, 2, ov);
    } else {
      if (gz > e.z) cp = box_feature_sphere(e, c, r, 6, 1, ov);
      else if (gz < -e.z) cp = box_feature_sphere(e, c, r, 1, 1, ov);
      else {
        nd = xsub(gx, e.x);
        if (nd < r) { *ov = xsub(nd, r); cp = d3(xadd(e.x, xmul(0.5, *ov)), c.y, c.z); }
      }
    }
  } else if (gx < -e.x) {
    if (gy > e.y) {
      if (gz > e.z) cp = box_feature_sphere(e, c, r, 7, -1, ov);
      else if (gz < -e.z) cp = box_feature_sphere(e, c, r, 4, -1, ov);
      else cp = box_feature_sphere(e, c, r, 4, 2, ov);
    } else if (gy < -e.y) {
      if (gz > e.z) cp = box_feature_sphere(e, c, r, 3, -1, ov);
      else if (gz < -e.z) cp = box_feature_sphere(e, c, r, 0, -1, ov);
      else cp = box_feature_sphere(e, c, r, 0, 2, ov);
    } else {
      if (gz > e.z) cp = box_feature_sphere(e, c, r, 3, 1, ov);
      else if (gz < -e.z) cp = box_feature_sphere(e, c, r, 0, 1, ov);
      else {
        nd = xsub(-e.x, gx);
        if (nd < r) { *ov = xsub(nd, r); cp = d3(xsub(-e.x, xmul(0.5, *ov)), c.y, c.z); }
      }
    }
  } else {
    if (gy > e.y) {
      if (gz > e.z) cp = box_feature_sphere(e, c, r, 6, 0, ov);
      else if (gz < -e.z) cp = box_feature_sphere(e, c, r, 4, 0, ov);
      else {
        nd = xsub(gy, e.y);
        if (nd < r) { *ov = xsub(nd, r); cp = d3(c.x, xadd(e.y, xmul(0.5, *ov)), c.z); }
      }
    } else if (gy < -e.y) {
      if (gz > e.z) cp = box_feature_sphere(e, c, r, 3, 0, ov);
      else if (gz < -e.z) cp = box_feature_sphere(e, c, r, 0, 0, ov);
      else {
        nd = xsub(-e.y, gy);
        if (nd < r) { *ov = xsub(nd, r); cp = d3(c.x, xsub(-e.y, xmul(0.5, *ov)), c.z); }
      }
    } else {
      if (gz > e.z) {
        nd = xsub(gz, e.z);
        if (nd < r) { *ov = xsub(nd, r); cp = d3(c.x, c.y, xadd(e.z, xmul(0.5, *ov))); }
      } else if (gz < -e.z) {
        nd = xsub(-e.z, gz);
        if (nd < r) { *ov = xsub(nd, r); cp = d3(c.x, c.y, xsub(-e.z, xmul(0.5, *ov))); }
      } else {
        *inside = 1;
        *ov = -10000.;
      }
    }
  }
  return cp;
}

// ClosestPointSPHEREBOX with the sphere as body A (the particle-wall case,
// SimpleObstacle::InterAction passes the particle first).  The box transform
// is basis b + origin o, never scaled; its inverse is the transpose
// (Transform::setToInverseTransform, Transform.cpp:52-58).
GG_HD ContactGeom sphere_box(D3 ca, double ra, double crust_sum, const M3& b, D3 o, D3 ext) {
  M3 bt = mtranspose(b);
  D3 io = d3(-xdot(mrow(bt, 0), o), -xdot(mrow(bt, 1), o), -xdot(mrow(bt, 2), o));
  D3 local = xapply(bt, io, ca);
  double ov;
  int inside;
  D3 cp = box_sphere_local(ext, local, ra, &ov, &inside);
  if (inside) {
    ContactGeom c = no_contact();
    c.status = 1;
    c.overlap = -1.e20;
    return c;
  }
  if (!(ov < 0.)) return no_contact();
  ContactGeom c;
  c.status = (-ov >= crust_sum) ? 1 : 0;
  c.point = xapply(b, o, cp);
  D3 ab = xsub3(c.point, ca);
  c.overlap_vector = xscale(ab, xdiv(ov, xnorm(ab)));
  c.overlap = ov;
  return c;
}

// BBox::InZone (Geometry/src/BBox.cpp:166-185)
GG_HD bool in_zone(D3 bc, D3 be, D3 p, double hx, double hy, double hz) {
  return std::fabs(xsub(bc.x, p.x)) <= xadd(be.x, hx) && std::fabs(xsub(bc.y, p.y)) <= xadd(be.y, hy) &&
         std::fabs(xsub(bc.z, p.z)) <= xadd(be.z, hz);
}

}  // namespace gg
