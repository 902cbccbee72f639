// Explicit dynamics driver written against the C++ drop-in API, in the shape
// of the reference's explicit examples: parse a material file, build or read
// a mesh, initFull(_analysis_method = _explicit_lumped_mass), block a face,
// set an initial velocity, step, report.
//
//   explicit_dynamic <material.dat> <hex8|tet4> <cells> <steps> [mixed]
//
// Prints one line "u_max <value> ekin <value> epot <value> steps <n>".
#include <akantu_b200/solid_mechanics_model.hh>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace akantu_b200;

// structured box [0,1]^3 of n^3 cells (hexahedra, or 6 tetrahedra per cell)
static void build_box(Mesh &mesh, bool hex, int n) {
  const int m = n + 1;
  Array<Real> nodes((Int)m * m * m, 3);
  for (int k = 0; k < m; ++k)
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) {
        const Int id = i + m * (j + m * k);
        nodes(id, 0) = (Real)i / n;
        nodes(id, 1) = (Real)j / n;
        nodes(id, 2) = (Real)k / n;
      }
  auto nid = [m](int i, int j, int k) { return (Idx)(i + m * (j + m * k)); };
  Array<Idx> conn(0, hex ? 8 : 4);
  std::vector<Idx> c;
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        if (hex) {
          Idx h[8] = {nid(i, j, k),         nid(i + 1, j, k),     nid(i + 1, j + 1, k),
                      nid(i, j + 1, k),     nid(i, j, k + 1),     nid(i + 1, j, k + 1),
                      nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)};
          c.insert(c.end(), h, h + 8);
        } else {
          // Kuhn split along the main diagonal, positively oriented
          const int perms[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
          for (int p = 0; p < 6; ++p) {
            int v[4][3] = {{i, j, k}};
            for (int s = 0; s < 3; ++s) {
              for (int d = 0; d < 3; ++d) v[s + 1][d] = v[s][d];
              v[s + 1][perms[p][s]] += 1;
            }
            Idx t[4];
            for (int s = 0; s < 4; ++s) t[s] = nid(v[s][0], v[s][1], v[s][2]);
            if (p >= 3) std::swap(t[1], t[2]);
            c.insert(c.end(), t, t + 4);
          }
        }
      }
  conn.resize((Int)c.size() / conn.getNbComponent());
  std::copy(c.begin(), c.end(), conn.data());
  mesh.setElements(hex ? _hexahedron_8 : _tetrahedron_4, nodes, conn);
}

int main(int argc, char *argv[]) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s material.dat hex8|tet4 cells steps [mixed]\n", argv[0]);
    return 2;
  }
  try {
    initialize(argv[1], argc, argv);
    Mesh mesh(3);
    build_box(mesh, std::string(argv[2]) == "hex8", std::atoi(argv[3]));
    const Int nsteps = std::atol(argv[4]);

    // z = 0 face: every component blocked
    std::vector<Idx> bottom;
    const auto &X = mesh.getNodes();
    for (Int n = 0; n < mesh.getNbNodes(); ++n)
      if (X(n, 2) == 0.) bottom.push_back((Idx)n);
    mesh.createNodeGroup("bottom", bottom);

    SolidMechanicsModel model(mesh);
    if (argc > 5 && std::string(argv[5]) == "mixed")
      model.initFullMixedPrecision();
    else
      model.initFull(_analysis_method = _explicit_lumped_mass);

    model.applyBC(BC::Dirichlet::FixedValue(0., _x), "bottom");
    model.applyBC(BC::Dirichlet::FixedValue(0., _y), "bottom");
    model.applyBC(BC::Dirichlet::FixedValue(0., _z), "bottom");

    // v_z = 0.01 sin(pi x) sin(pi y) z
    auto &v = model.getVelocity();
    for (Int n = 0; n < mesh.getNbNodes(); ++n)
      v(n, 2) = 0.01 * std::sin(M_PI * X(n, 0)) * std::sin(M_PI * X(n, 1)) * X(n, 2);

    model.setTimeStep(0.8 * model.getStableTimeStep());
    for (Int s = 0; s < nsteps; ++s) model.solveStep();

    const auto &u = model.getDisplacement();
    Real umax = 0.;
    for (Int k = 0; k < u.size() * 3; ++k) umax = std::fmax(umax, std::fabs(u.data()[k]));
    std::printf("u_max %.17g ekin %.17g epot %.17g steps %lld\n", umax,
                model.getEnergy("kinetic"), model.getEnergy("potential"), (long long)nsteps);
  } catch (const Exception &e) {
    std::fprintf(stderr, "error %d: %s\n", e.code(), e.what());
    return 1;
  }
  return 0;
}
