// elem_shapes.cuh -- reference-element data of the quadrature-integrated edge
// elements (HEX8_EDGE, PRISM6_EDGE, PYRAMID5_EDGE, and TET4_EDGE inside mixed
// meshes): Lagrange map, edge basis and its
// reference curl, quadrature.  Each shape is a struct of constexpr sizes and
// __host__ __device__ functions, so the same definitions serve the assembly
// kernels and their host-side tests.
//
// Conventions shared by the shapes (MagneticVector3DIntegrator,
// magnetic_vector_3d_integrator.cpp:139-364):
//   J[r][c] = sum_a X_a[r] dN_a/dx_c,  curl_phys = J curl_ref / det J,
//   W_phys = J^-T W_ref,  K_ij = sum_q w_q |det J| nu curl_i . curl_j, ...
// Edge k runs from local node a to b of ElementGeometry's table
// (element_geometry.cpp:161-181 HEX8, :214-237 PRISM6, :268-289 PYRAMID5);
// the prism and pyramid bases have unit circulation along a -> b and none
// along the other edges.
#pragma once

namespace emg {
namespace shape {

// ------------------------------------------------------------------ TET4 ----
// The reference's Whitney tetrahedron in a mixed mesh (a mesh of tets alone
// takes k_tet_terms): N_0 = xi, N_1 = eta, N_2 = zeta, N_3 = 1 - xi - eta -
// zeta (lagrange_element.cpp:658-683); local edge k (ElementGeometry's
// {0,1},{1,2},{0,2},{0,3},{1,3},{2,3}) carries the function of the Nedelec
// pair (p, q) = {0,1},{1,2},{2,0},{0,3},{1,3},{2,3} (nedelec_element.cpp:54-60,
// :411-505): N_q grad N_p - N_p grad N_q, which circulates from q to p, so
// edge_a = q, edge_b = p; its curl is 2 grad N_q x grad N_p (the constant
// curls of curlTet4Edge).  Hammer 4-point rule, weights 1/24
// (gauss_quadrature.cpp:184-227 with its fourth point).
struct Tet {
  static constexpr int kType = 0, kNodes = 4, kEdges = 6, kPoints = 4;
  __host__ __device__ static constexpr int ned_p(int k) { return k < 3 ? k : k - 3; }
  __host__ __device__ static constexpr int ned_q(int k) { return k < 3 ? (k + 1) % 3 : 3; }
  __host__ __device__ static constexpr int edge_a(int k) { return ned_q(k); }
  __host__ __device__ static constexpr int edge_b(int k) { return ned_p(k); }
  __host__ __device__ static double dcoord(int a, int c) { return a == 3 ? -1.0 : (a == c ? 1.0 : 0.0); }
  __host__ __device__ static void point(int q, double* x, double* w) {
    const double qa = 0.13819660112501051517954131656343619;  // (5 - sqrt 5) / 20
    const double qb = 0.58541019662496845446137605030969143;  // (5 + 3 sqrt 5) / 20
    x[0] = q == 2 ? qb : qa;
    x[1] = q == 1 ? qb : qa;
    x[2] = q == 0 ? qb : qa;
    *w = 1.0 / 24.0;
  }
  __host__ __device__ static double n(int a, const double* x) { return a == 3 ? 1.0 - x[0] - x[1] - x[2] : x[a]; }
  __host__ __device__ static void dn(int a, const double* x, double* d) {
    (void)x;
    for (int c = 0; c < 3; ++c) d[c] = dcoord(a, c);
  }
  __host__ __device__ static void basis(int k, const double* x, double* w) {
    const int p = ned_p(k), q = ned_q(k);
    const double np = n(p, x), nq = n(q, x);
    for (int c = 0; c < 3; ++c) w[c] = nq * dcoord(p, c) - np * dcoord(q, c);
  }
  __host__ __device__ static void curl(int k, const double* x, double* c) {
    (void)x;
    const int p = ned_p(k), q = ned_q(k);
    c[0] = 2.0 * (dcoord(q, 1) * dcoord(p, 2) - dcoord(q, 2) * dcoord(p, 1));
    c[1] = 2.0 * (dcoord(q, 2) * dcoord(p, 0) - dcoord(q, 0) * dcoord(p, 2));
    c[2] = 2.0 * (dcoord(q, 0) * dcoord(p, 1) - dcoord(q, 1) * dcoord(p, 0));
  }
};

// ------------------------------------------------------------------ HEX8 ----
// Reference hexahedron [-1,1]^3, nodes 0-3 on zeta = -1 (counter-clockwise
// from (-1,-1)), 4-7 above them (nedelec_element.cpp:506-517; HEX8 map
// N_a = 1/8 prod (1 + c_a x), lagrange_element.cpp:765-772).  Edge k runs
// from local node A to B (ElementGeometry's table, element_geometry.cpp:165-171)
// along reference axis d; with (p, q) = (d+1, d+2) mod 3 and c_p, c_q the
// edge's fixed coordinates, its basis (evalHex8Edge, nedelec_element.cpp:519-615) is
//   W_k = 1/2 s_k (1 + c_p x_p)(1 + c_q x_q) e_d,   s_k = (x_d(B) - x_d(A)) / 2,
// (circulation 4 along its edge: the reference's normalisation) with curl
//   curl W_k = 1/2 s_k [c_q (1 + c_p x_p) e_p - c_p (1 + c_q x_q) e_q].
// (curlHex8Edge, :618-720, has sign / component errors in edges 2, 3, 6, 7;
// the curl here is the derivative of the reference's own W_k.)  Quadrature:
// 2x2x2 Gauss-Legendre, weights 1, xi outermost (getHex8Points,
// gauss_quadrature.cpp:247-276).
struct Hex {
  static constexpr int kType = 1, kNodes = 8, kEdges = 12, kPoints = 8;
  __host__ __device__ static constexpr int coord(int a, int axis) {  // reference coordinate of node a
    return axis == 0 ? (((a & 3) == 1 || (a & 3) == 2) ? 1 : -1) : axis == 1 ? ((a & 2) ? 1 : -1) : ((a & 4) ? 1 : -1);
  }
  __host__ __device__ static constexpr int edge_a(int k) { return k < 8 ? k : k - 8; }
  __host__ __device__ static constexpr int edge_b(int k) {
    return k < 4 ? ((k + 1) & 3) : k < 8 ? 4 + ((k + 1) & 3) : k - 4;
  }
  __host__ __device__ static constexpr int dir(int k) { return k < 8 ? (k & 1) : 2; }
  __host__ __device__ static constexpr int sgn(int k) { return (coord(edge_b(k), dir(k)) - coord(edge_a(k), dir(k))) / 2; }
  __host__ __device__ static constexpr int cp(int k) { return coord(edge_a(k), (dir(k) + 1) % 3); }
  __host__ __device__ static constexpr int cq(int k) { return coord(edge_a(k), (dir(k) + 2) % 3); }
  __host__ __device__ static void point(int q, double* x, double* w) {
    const double g = 0.57735026918962576450914878050195746;  // 1 / sqrt 3
    x[0] = (q & 4) ? g : -g;
    x[1] = (q & 2) ? g : -g;
    x[2] = (q & 1) ? g : -g;
    *w = 1.0;
  }
  __host__ __device__ static double n(int a, const double* x) {
    return 0.125 * (1.0 + coord(a, 0) * x[0]) * (1.0 + coord(a, 1) * x[1]) * (1.0 + coord(a, 2) * x[2]);
  }
  __host__ __device__ static void dn(int a, const double* x, double* d) {
    const double l0 = 1.0 + coord(a, 0) * x[0], l1 = 1.0 + coord(a, 1) * x[1], l2 = 1.0 + coord(a, 2) * x[2];
    d[0] = 0.125 * coord(a, 0) * l1 * l2;
    d[1] = 0.125 * coord(a, 1) * l0 * l2;
    d[2] = 0.125 * coord(a, 2) * l0 * l1;
  }
  __host__ __device__ static void basis(int k, const double* x, double* w) {
    const int d = dir(k), p = (d + 1) % 3, q = (d + 2) % 3;
    w[0] = w[1] = w[2] = 0.0;
    w[d] = 0.5 * sgn(k) * (1.0 + cp(k) * x[p]) * (1.0 + cq(k) * x[q]);
  }
  __host__ __device__ static void curl(int k, const double* x, double* c) {
    const int d = dir(k), p = (d + 1) % 3, q = (d + 2) % 3;
    c[d] = 0.0;
    c[p] = 0.5 * sgn(k) * cq(k) * (1.0 + cp(k) * x[p]);
    c[q] = -0.5 * sgn(k) * cp(k) * (1.0 + cq(k) * x[q]);
  }
};
static_assert(Hex::edge_a(2) == 2 && Hex::edge_b(2) == 3 && Hex::edge_b(3) == 0 && Hex::edge_b(7) == 4 &&
                  Hex::edge_b(11) == 7,
              "edge table of element_geometry.cpp:165-171");
static_assert(Hex::sgn(2) == -1 && Hex::sgn(3) == -1 && Hex::sgn(6) == -1 && Hex::sgn(7) == -1 && Hex::sgn(8) == 1,
              "basis orientation of nedelec_element.cpp:519-615");
static_assert(Hex::cp(0) == -1 && Hex::cq(0) == -1 && Hex::cp(1) == -1 && Hex::cq(1) == 1 && Hex::cp(9) == 1 &&
                  Hex::cq(9) == -1,
              "edge positions");

// ---------------------------------------------------------------- PRISM6 ----
// Reference prism: triangle xi, eta >= 0, xi + eta <= 1, zeta in [-1, 1].
// Nodes by the reference's PRISM6 Lagrange functions
// (lagrange_element.cpp:458-522): node a (a < 3) has area coordinate
// L_a (L_0 = xi, L_1 = eta, L_2 = 1 - xi - eta) at zeta = -1, node a + 3 the
// same at zeta = +1; N_a = L_a (1 - zeta) / 2, N_{a+3} = L_a (1 + zeta) / 2.
// Basis (the forms of evalPrism6Edge, nedelec_element.cpp:744-792, with each
// function on its own edge): bottom edge (a, b): h(zeta) (L_a grad L_b -
// L_b grad L_a), h = (1 - zeta) / 2; top edges the same with h = (1 + zeta)
// / 2; vertical edge (a, a + 3): L_a grad(zeta) / 2.  Quadrature: the
// reference's 3-point triangle rule x 2-point Gauss in zeta
// (GaussQuadrature::getPrism6Points, gauss_quadrature.cpp:304-345).
struct Prism {
  static constexpr int kType = 2, kNodes = 6, kEdges = 9, kPoints = 6;
  __host__ __device__ static constexpr int edge_a(int k) { return k < 3 ? (k == 2 ? 0 : k) : k < 6 ? (k == 5 ? 3 : k) : k - 6; }
  __host__ __device__ static constexpr int edge_b(int k) {
    return k < 3 ? (k == 0 ? 1 : 2) : k < 6 ? (k == 3 ? 4 : 5) : k - 3;
  }
  // area coordinate of triangle vertex a and its (xi, eta) gradient
  __host__ __device__ static double area(int a, double xi, double eta) {
    return a == 0 ? xi : a == 1 ? eta : 1.0 - xi - eta;
  }
  __host__ __device__ static double darea(int a, int c) {  // d L_a / d(xi, eta)[c]
    return a == 0 ? (c == 0 ? 1.0 : 0.0) : a == 1 ? (c == 0 ? 0.0 : 1.0) : -1.0;
  }
  __host__ __device__ static void point(int q, double* x, double* w) {
    const double g = 0.57735026918962576450914878050195746;  // 1 / sqrt 3
    const int it = q % 3, iz = q / 3;
    x[0] = it == 1 ? 2.0 / 3.0 : 1.0 / 6.0;
    x[1] = it == 2 ? 2.0 / 3.0 : 1.0 / 6.0;
    x[2] = iz == 0 ? -g : g;
    *w = 1.0 / 6.0;
  }
  __host__ __device__ static double n(int a, const double* x) {
    const double h = a < 3 ? 0.5 * (1.0 - x[2]) : 0.5 * (1.0 + x[2]);
    return area(a % 3, x[0], x[1]) * h;
  }
  __host__ __device__ static void dn(int a, const double* x, double* d) {
    const int v = a % 3;
    const double h = a < 3 ? 0.5 * (1.0 - x[2]) : 0.5 * (1.0 + x[2]);
    d[0] = h * darea(v, 0);
    d[1] = h * darea(v, 1);
    d[2] = (a < 3 ? -0.5 : 0.5) * area(v, x[0], x[1]);
  }
  __host__ __device__ static void basis(int k, const double* x, double* w) {
    if (k < 6) {
      const int a = edge_a(k) % 3, b = edge_b(k) % 3;
      const double h = k < 3 ? 0.5 * (1.0 - x[2]) : 0.5 * (1.0 + x[2]);
      const double la = area(a, x[0], x[1]), lb = area(b, x[0], x[1]);
      w[0] = h * (la * darea(b, 0) - lb * darea(a, 0));
      w[1] = h * (la * darea(b, 1) - lb * darea(a, 1));
      w[2] = 0.0;
    } else {
      w[0] = 0.0;
      w[1] = 0.0;
      w[2] = 0.5 * area(k - 6, x[0], x[1]);
    }
  }
  // curl (h w) = h' e_zeta x w + h curl w, curl w = 2 grad L_a x grad L_b;
  // curl (L_a e_zeta / 2) = grad(L_a) x e_zeta / 2
  __host__ __device__ static void curl(int k, const double* x, double* c) {
    if (k < 6) {
      const int a = edge_a(k) % 3, b = edge_b(k) % 3;
      const double h = k < 3 ? 0.5 * (1.0 - x[2]) : 0.5 * (1.0 + x[2]);
      const double dh = k < 3 ? -0.5 : 0.5;
      const double la = area(a, x[0], x[1]), lb = area(b, x[0], x[1]);
      const double wx = la * darea(b, 0) - lb * darea(a, 0);
      const double wy = la * darea(b, 1) - lb * darea(a, 1);
      c[0] = -dh * wy;
      c[1] = dh * wx;
      c[2] = 2.0 * h * (darea(a, 0) * darea(b, 1) - darea(a, 1) * darea(b, 0));
    } else {
      const int a = k - 6;
      c[0] = 0.5 * darea(a, 1);
      c[1] = -0.5 * darea(a, 0);
      c[2] = 0.0;
    }
  }
};

// -------------------------------------------------------------- PYRAMID5 ----
// Reference pyramid as the reference's PYRAMID5 Lagrange map writes it
// (lagrange_element.cpp:51-135): xi, eta in [-1, 1], zeta in [0, 1],
// N_a = (1 - zeta) P_a(xi, eta) for the base corners a = 0..3 at
// (-1,-1), (1,-1), (1,1), (-1,1) (P_a bilinear), N_4 = zeta: the cube
// collapsed onto the apex at zeta = 1 (in physical coordinates the rational
// pyramid functions).  Basis (H(curl)-conforming: tangential traces equal
// the tetrahedron's Whitney functions on the four triangular faces and a
// unit-circulation hexahedron's bilinear edge functions on the base; the
// gradients of N_0..N_4 lie in the span):
//   base edge a -> a+1 along +-e_d:  W = 1/4 (1 + c_perp x_perp) (1 - zeta)^2 (+-e_d)
//   slant edge a -> apex:            W = N_a grad N_4 - N_4 grad N_a
//                                      = P_a e_zeta - zeta (1 - zeta) grad P_a
// (evalPyramid5Edge, nedelec_element.cpp:854-990, has base functions that do
// not vanish tangentially on the triangular faces).  Quadrature: 2 x 2
// Gauss-Legendre in xi, eta x 3-point Gauss-Legendre in zeta on [0, 1],
// exact for the integrands of an affine pyramid (the reference's 5-point
// rule, gauss_quadrature.cpp:380-433, is stated on zeta in [-1, 1] with
// weights summing to 4/3).
struct Pyramid {
  static constexpr int kType = 3, kNodes = 5, kEdges = 8, kPoints = 12;
  __host__ __device__ static constexpr int edge_a(int k) { return k < 4 ? k : k - 4; }
  __host__ __device__ static constexpr int edge_b(int k) { return k < 4 ? (k + 1) & 3 : 4; }
  __host__ __device__ static double cx(int a) { return (a == 1 || a == 2) ? 1.0 : -1.0; }
  __host__ __device__ static double cy(int a) { return a >= 2 ? 1.0 : -1.0; }
  __host__ __device__ static double p(int a, double xi, double eta) {
    return 0.25 * (1.0 + cx(a) * xi) * (1.0 + cy(a) * eta);
  }
  __host__ __device__ static double px(int a, double eta) { return 0.25 * cx(a) * (1.0 + cy(a) * eta); }
  __host__ __device__ static double py(int a, double xi) { return 0.25 * cy(a) * (1.0 + cx(a) * xi); }
  __host__ __device__ static void point(int q, double* x, double* w) {
    const double g = 0.57735026918962576450914878050195746;  // 1 / sqrt 3
    const double s = 0.77459666924148337703585307995647992;  // sqrt(3 / 5)
    const int iz = q % 3, ie = (q / 3) & 1, ix = q / 6;
    x[0] = ix ? g : -g;
    x[1] = ie ? g : -g;
    x[2] = 0.5 * (1.0 + (iz == 0 ? -s : iz == 1 ? 0.0 : s));
    *w = 0.5 * (iz == 1 ? 8.0 / 9.0 : 5.0 / 9.0);
  }
  __host__ __device__ static double n(int a, const double* x) {
    return a == 4 ? x[2] : (1.0 - x[2]) * p(a, x[0], x[1]);
  }
  __host__ __device__ static void dn(int a, const double* x, double* d) {
    if (a == 4) {
      d[0] = 0.0;
      d[1] = 0.0;
      d[2] = 1.0;
    } else {
      d[0] = (1.0 - x[2]) * px(a, x[1]);
      d[1] = (1.0 - x[2]) * py(a, x[0]);
      d[2] = -p(a, x[0], x[1]);
    }
  }
  __host__ __device__ static void basis(int k, const double* x, double* w) {
    const double r = 1.0 - x[2];
    if (k < 4) {
      w[0] = w[1] = w[2] = 0.0;
      if (k == 0) w[0] = 0.25 * (1.0 - x[1]) * r * r;
      else if (k == 1) w[1] = 0.25 * (1.0 + x[0]) * r * r;
      else if (k == 2) w[0] = -0.25 * (1.0 + x[1]) * r * r;
      else w[1] = -0.25 * (1.0 - x[0]) * r * r;
    } else {
      const int a = k - 4;
      const double g = x[2] * r;
      w[0] = -g * px(a, x[1]);
      w[1] = -g * py(a, x[0]);
      w[2] = p(a, x[0], x[1]);
    }
  }
  __host__ __device__ static void curl(int k, const double* x, double* c) {
    const double r = 1.0 - x[2];
    if (k < 4) {
      c[2] = 0.25 * r * r;
      if (k == 0) { c[0] = 0.0; c[1] = -0.5 * (1.0 - x[1]) * r; }
      else if (k == 1) { c[0] = 0.5 * (1.0 + x[0]) * r; c[1] = 0.0; }
      else if (k == 2) { c[0] = 0.0; c[1] = 0.5 * (1.0 + x[1]) * r; }
      else { c[0] = -0.5 * (1.0 - x[0]) * r; c[1] = 0.0; }
    } else {
      const int a = k - 4;
      c[0] = 2.0 * r * py(a, x[0]);
      c[1] = -2.0 * r * px(a, x[1]);
      c[2] = 0.0;
    }
  }
};

}  // namespace shape
}  // namespace emg
