// A solve service in C++: hexahedral boxes of several sizes are submitted to
// the server (akantu_b200::Server over akb_server_*), which keeps them
// resident on the GPU and advances them together; the driver polls the
// completions and prints each solve's latency and the maximum displacement.
//
//   serve_boxes <requests> <steps>
//
// Prints one line per solve "id <id> elements <E> latency_s <t> u_max <u>".
#include <akantu_b200/solid_mechanics_model.hh>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <vector>

using namespace akantu_b200;

namespace {

struct Box {
  int n = 0;
  std::vector<double> nodes, v, u;
  std::vector<int32_t> conn;
  std::vector<uint8_t> blocked;
};

// n^3 hexahedra on [0,1]^3, z = 0 blocked, a sinusoidal initial velocity
Box make_box(int n) {
  Box b;
  b.n = n;
  const int m = n + 1;
  for (int k = 0; k < m; ++k)
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) {
        const double x = (double)i / n, y = (double)j / n, z = (double)k / n;
        b.nodes.insert(b.nodes.end(), {x, y, z});
        b.v.insert(b.v.end(), {0., 0., 0.01 * std::sin(M_PI * x) * std::sin(M_PI * y) * z});
        const uint8_t fixed = k == 0 ? 1 : 0;
        b.blocked.insert(b.blocked.end(), {fixed, fixed, fixed});
      }
  auto id = [m](int i, int j, int k) { return (int32_t)(i + m * (j + m * k)); };
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        b.conn.insert(b.conn.end(),
                      {id(i, j, k), id(i + 1, j, k), id(i + 1, j + 1, k), id(i, j + 1, k),
                       id(i, j, k + 1), id(i + 1, j, k + 1), id(i + 1, j + 1, k + 1),
                       id(i, j + 1, k + 1)});
  b.u.assign(b.nodes.size(), 0.);
  return b;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <requests> <steps>\n", argv[0]);
    return 2;
  }
  const int requests = std::atoi(argv[1]);
  const int64_t steps = std::atoll(argv[2]);
  try {
    akb_server_config cfg{};
    cfg.max_active = 16;
    Server server(cfg);
    std::vector<Box> boxes;
    boxes.reserve(requests);
    std::map<int64_t, size_t> box_of;
    for (int r = 0; r < requests; ++r) {
      boxes.push_back(make_box(4 + 4 * (r % 4)));
      Box &b = boxes.back();
      akb_request q{};
      q.element_type = AKB_HEXAHEDRON_8;
      q.precision = AKB_PRECISION_MIXED;
      q.nb_nodes = (int64_t)b.nodes.size() / 3;
      q.nb_elements = (int64_t)b.conn.size() / 8;
      q.nodes = b.nodes.data();
      q.connectivity = b.conn.data();
      q.material_type = "neohookean";
      q.material_params = "rho = 1; E = 1; nu = 0.3";
      q.velocity = b.v.data();
      q.blocked_dofs = b.blocked.data();
      q.dt_factor = 0.8;
      q.nb_steps = steps;
      q.displacement_out = b.u.data();
      box_of[server.submit(q)] = boxes.size() - 1;
    }
    int done = 0;
    while (done < requests) {
      for (const akb_completion &c : server.poll(0.05)) {
        ++done;
        const Box &b = boxes[box_of.at(c.id)];
        double umax = 0.;
        for (double x : b.u) umax = std::max(umax, std::fabs(x));
        if (c.status != AKB_OK) {
          std::printf("id %lld failed %d %s\n", (long long)c.id, c.status, c.message);
          continue;
        }
        std::printf("id %lld elements %lld latency_s %.4f u_max %.6e\n", (long long)c.id,
                    (long long)c.nb_elements, c.t_end - c.t_submit, umax);
      }
    }
  } catch (const Exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
