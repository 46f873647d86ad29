// Tests of the clue:: C++ API (include/CLUEstering) over libclue_b200.
//
//   test_api cpu <scratch_dir>
//       host-only parts: kernel and metric objects, points containers, association maps,
//       cluster properties, CSV I/O, centroids.  Needs no GPU.
//   test_api gpu <input.csv> <dc> <rhoc> <dm> <output.csv>
//       clusters a 2-D CSV through every make_clusters overload and the device containers,
//       checks that they agree with one another, that host and device association maps match,
//       and writes x0,x1,weight,cluster_id,is_seed,nearest_higher,rho_bits,delta_bits plus a
//       summary line "silhouette=<s> n_clusters=<k>" to stdout for the caller to compare with
//       the oracle.
// Modelled on the reference's C++ tests (tests/test_clusterer.cpp, test_host_points.cpp,
// test_device_points.cpp, test_association_map.cpp, test_convolutional_kernels.cpp,
// test_distance_metrics.cpp, test_cluster_centroid.cpp).
#include "CLUEstering/CLUEstering.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <numeric>
#include <ranges>
#include <string>
#include <vector>

static int g_failures = 0;
#define CHECK(cond)                                                            \
  do {                                                                         \
    if (!(cond)) {                                                             \
      std::fprintf(stderr, "FAIL %s:%d: %s\n", __FILE__, __LINE__, #cond);     \
      ++g_failures;                                                            \
    }                                                                          \
  } while (0)
#define CHECK_THROWS_AS(expr, type)                                            \
  do {                                                                         \
    bool thrown_ = false;                                                      \
    try {                                                                      \
      (void)(expr);                                                            \
    } catch (const type&) {                                                    \
      thrown_ = true;                                                          \
    } catch (...) {                                                            \
    }                                                                          \
    if (!thrown_) {                                                            \
      std::fprintf(stderr, "FAIL %s:%d: %s does not throw %s\n", __FILE__,    \
                   __LINE__, #expr, #type);                                    \
      ++g_failures;                                                            \
    }                                                                          \
  } while (0)

static uint32_t bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

// ---------------------------------------------------------------------------------------------
static void test_kernels() {
  CHECK_THROWS_AS(clue::FlatKernel(0.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::FlatKernel(-1.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::ExponentialKernel(0.f, 1.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::ExponentialKernel(1.f, 0.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::ExponentialKernel(-1.f, 1.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::ExponentialKernel(1.f, -1.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::GaussianKernel(1.f, 0.f, 1.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::GaussianKernel(1.f, 1.f, 0.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::GaussianKernel(-1.f, 1.f, 1.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::GaussianKernel(1.f, -1.f, 1.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::GaussianKernel(1.f, 1.f, -1.f), std::invalid_argument);
  // mean 0 is accepted (a deliberate widening of the reference's check)
  clue::GaussianKernel g0(0.f, 0.5f, 1.f);
  CHECK(g0(0.f, 1, 2) == 1.f);
  clue::FlatKernel flat(.5f);
  CHECK(flat(0.3f, 4, 4) == 1.f);
  CHECK(flat(0.3f, 4, 5) == .5f);
  clue::ExponentialKernel ek(1.f, 2.f);
  CHECK(ek(0.f, 0, 0) == 1.f);
  CHECK(std::fabs(ek(1.f, 0, 1) - 2.f * std::exp(-1.f)) < 1e-6f);
}

static void test_metrics() {
  clue::Point<2> a{0.f, 0.f, 7.f}, b{3.f, 4.f, 9.f};
  CHECK(clue::EuclideanMetric<2>{}(a, b) == 5.f);
  CHECK(clue::metrics::Manhattan<2>{}(a, b) == 7.f);
  CHECK(clue::metrics::Chebyshev<2>{}(a, b) == 4.f);
  CHECK(clue::WeightedEuclideanMetric<2>(1.f, 0.f)(a, b) == 3.f);
  CHECK(clue::WeightedChebyshevMetric<2>(2.f, 1.f)(a, b) == 6.f);
  clue::PeriodicEuclideanMetric<2> per(std::array<float, 2>{10.f, 0.f});
  clue::Point<2> c{9.f, 0.f, 1.f};
  CHECK(per(a, c) == 1.f);  // |9 - 0| wraps to 1 with period 10
  clue::Point<3> p3{1.f, 2.f, 2.f, 0.f}, o3{0.f, 0.f, 0.f, 0.f};
  CHECK(clue::EuclideanMetric<3>{}(p3, o3) == 3.f);
  static_assert(clue::concepts::distance_metric<clue::EuclideanMetric<2>, 2>);
}

static void test_host_points() {
  const int32_t size = 1000;
  auto dim = clue::Dim<2>{};
  CHECK_THROWS_AS(clue::PointsHost(dim, 0), std::invalid_argument);
  CHECK_THROWS_AS(clue::PointsHost(dim, -5), std::invalid_argument);
  {
    clue::PointsHost points(dim, size);
    CHECK(points.size() == size);
    std::iota(points.coords(0).begin(), points.coords(1).end(), 0.f);  // owned buffer is one SoA block
    std::fill(points.weights().begin(), points.weights().end(), 1.f);
    CHECK(points[0][0] == 0.f && points[0][1] == 1000.f && points[0].weight() == 1.f);
    CHECK(points[999][0] == 999.f && points[999][1] == 1999.f);
    CHECK_THROWS_AS(points[1000], std::out_of_range);
    CHECK_THROWS_AS(points.coords(3), std::out_of_range);
    const auto& cp = points;
    CHECK_THROWS_AS(cp.coords(10), std::out_of_range);
    CHECK(!points.clustered());
  }
  std::vector<float> coords(2 * size), weights(size), input(3 * size);
  std::vector<int> ids(size);
  std::vector<std::byte> whole(clue::PointsHost<2>::soa_bytes(size));
  {
    clue::PointsHost p(dim, size, std::span<std::byte>(whole));
    CHECK(reinterpret_cast<std::byte*>(p.view().coords[0]) == whole.data());
    CHECK(p.view().cluster_index == reinterpret_cast<int*>(whole.data() + 3 * size * sizeof(float)));
  }
  {
    clue::PointsHost p(dim, size, std::span<float>(input), std::span<int>(ids));
    CHECK(p.view().coords[1] == input.data() + size && p.view().weight == input.data() + 2 * size);
    CHECK(p.view().cluster_index == ids.data() && p.view().n == size);
  }
  {
    clue::PointsHost p(dim, size, std::span<float>(coords), std::span<float>(weights), std::span<int>(ids));
    CHECK(p.view().coords[1] == coords.data() + size && p.view().weight == weights.data());
  }
  {
    clue::PointsHost p(dim, size, input.data(), ids.data());
    CHECK(p.view().weight == input.data() + 2 * size);
  }
  {
    clue::PointsHost p(dim, size, coords.data(), weights.data(), ids.data());
    std::fill(p.weights().begin(), p.weights().end(), 2.f);
    CHECK(weights[17] == 2.f);
  }
  {
    std::vector<float> x(size), y(size);
    clue::PointsHost p(dim, size, x.data(), y.data(), weights.data(), ids.data());
    CHECK(p.view().coords[0] == x.data() && p.view().coords[1] == y.data() && p.view().weight == weights.data());
    clue::PointsHost q(dim, size, x, y, weights, ids);
    CHECK(q.view().coords[1] == y.data() && q.view().cluster_index == ids.data());
  }
}

static void test_association_map() {
  const int32_t size = 1000;
  std::vector<int32_t> assoc(size);
  for (int i = 0; i < size; ++i) assoc[i] = (i % 2 == 0);
  auto map = clue::internal::make_associator(std::span<const int32_t>(assoc), size);
  CHECK(map.size() == 2);
  CHECK(map.extents().values == (std::size_t)size && map.extents().keys == 2);
  CHECK(map.contains(0) && map.contains(1));
  CHECK(map.count(0) == (std::size_t)size / 2 && map.count(1) == (std::size_t)size / 2);
  CHECK(std::distance(map.begin(), map.end()) == size);
  CHECK(std::distance(map.lower_bound(0), map.upper_bound(0)) == size / 2);
  CHECK(std::distance(map.equal_range(1).first, map.equal_range(1).second) == size / 2);
  auto containers = map.extract();
  CHECK(containers.keys[0] == 0 && containers.keys[1] == size / 2 && containers.keys[2] == size);
  CHECK(containers.values[0] % 2 != 0 && containers.values[size - 1] % 2 == 0);
  // values ascend inside a key
  CHECK(std::is_sorted(map.lower_bound(0), map.upper_bound(0)));
  CHECK_THROWS_AS(map.count(-1), std::out_of_range);
  CHECK_THROWS_AS(map.count(2), std::out_of_range);
  CHECK_THROWS_AS(map.contains(3), std::out_of_range);
  CHECK_THROWS_AS(map.lower_bound(2), std::out_of_range);
  CHECK_THROWS_AS(map.upper_bound(-1), std::out_of_range);
  CHECK_THROWS_AS(map.equal_range(2), std::out_of_range);
  CHECK_THROWS_AS(clue::internal::make_associator(std::span<const int32_t>(assoc.data(), 0), 0),
                  std::invalid_argument);
  // outliers (-1) are left out
  std::vector<int32_t> with_outliers{-1, 2, 0, -1, 2, 2};
  auto m2 = clue::internal::make_associator(std::span<const int32_t>(with_outliers), 4);
  CHECK(m2.size() == 3 && m2.count(0) == 1 && m2.count(1) == 0 && m2.count(2) == 3);
  CHECK(*m2.lower_bound(2) == 1 && *(m2.upper_bound(2) - 1) == 5);
}

static void test_properties_io(const std::string& dir) {
  auto dim = clue::Dim<2>{};
  const std::string in = dir + "/points.csv";
  {
    std::ofstream f(in);
    f << "x0,x1,weight\n";
    for (int i = 0; i < 6; ++i) f << i << "," << 2 * i << ",1.5\n";
  }
  auto points = clue::read_csv(dim, in);
  CHECK(points.size() == 6 && points.coords(1)[5] == 10.f && points.weights()[3] == 1.5f && !points.clustered());
  CHECK_THROWS_AS(clue::read_csv(dim, dir + "/does_not_exist.csv"), std::runtime_error);
  const std::string out = dir + "/output.csv";
  {
    std::ofstream f(out);
    f << "x0,x1,weight,cluster_ids,is_seed\n";
    const int labels[6] = {0, 0, 1, -1, 1, 1};
    for (int i = 0; i < 6; ++i) f << i << "," << 2 * i << ",1," << labels[i] << "," << (i == 0) << "\n";
  }
  auto res = clue::read_output(dim, out);
  CHECK(res.clustered());
  CHECK(res.clusterIndexes()[3] == -1 && res.clusterIndexes()[5] == 1);
  CHECK(res.n_clusters() == 2);
  CHECK(res.clusters().size() == 2);
  CHECK(res.cluster_sizes().size() == 2 && res.cluster_sizes()[0] == 2 && res.cluster_sizes()[1] == 3);
  auto c1 = clue::cluster_centroid(res, 1);
  CHECK(std::fabs(c1[0] - 11.f / 3.f) < 1e-6f && std::fabs(c1[1] - 22.f / 3.f) < 1e-6f);
  auto cs = clue::cluster_centroids(res);
  CHECK(cs.size() == 2 && cs[0][0] == .5f && cs[0][1] == 1.f);
  auto gm = clue::get_clusters(res);
  CHECK(gm.size() == 2 && gm.count(1) == 3);
  const float s = clue::silhouette(res);
  CHECK(std::isfinite(s) && s > -1.f && s <= 1.f);
  // validate_results: cluster count and sizes, whatever the labels
  auto write_labels = [&](const std::string& path, const int (&labels)[6]) {
    std::ofstream f(path);
    f << "x0,x1,weight,cluster_ids,is_seed\n";
    for (int i = 0; i < 6; ++i) f << i << "," << 2 * i << ",1," << labels[i] << ",0\n";
  };
  const int relabelled[6] = {1, 1, 0, -1, 0, 0};
  const int moved[6] = {0, 0, 1, -1, -1, 1};
  const int merged[6] = {0, 0, 0, -1, 0, 0};
  write_labels(dir + "/relabelled.csv", relabelled);
  write_labels(dir + "/moved.csv", moved);
  write_labels(dir + "/merged.csv", merged);
  auto same = clue::read_output(dim, out);
  auto rel = clue::read_output(dim, dir + "/relabelled.csv");
  auto mov = clue::read_output(dim, dir + "/moved.csv");
  auto mer = clue::read_output(dim, dir + "/merged.csv");
  CHECK(clue::validate_results(res, same));
  CHECK(clue::validate_results(res, rel) && clue::validate_results(rel, res));
  CHECK(!clue::validate_results(res, mov));  // same count, sizes {2, 3} against {2, 2}
  CHECK(!clue::validate_results(res, mer));  // one cluster against two
}

// ---------------------------------------------------------------------------------------------
template <typename T>
static std::vector<T> to_host(std::span<const T> d) {
  std::vector<T> h(d.size());
  clue::detail::check(clue_memcpy_dtoh(h.data(), d.data(), d.size() * sizeof(T), nullptr));
  return h;
}

static int run_gpu(const std::string& in, float dc, float rhoc, float dm, const std::string& out) {
  auto device = clue::DevicePool::deviceAt(0u);
  auto& queue = clue::get_queue(device);
  clue::Dim<2> dim{};
  CHECK_THROWS_AS(clue::Clusterer(queue, dim, -1.f, 10.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::Clusterer(queue, dim, 1.f, -10.f), std::invalid_argument);
  CHECK_THROWS_AS(clue::Clusterer(queue, dim, 1.f, 1.f, 0.f), std::invalid_argument);

  clue::PointsHost h_points = clue::read_csv(dim, in);
  const int32_t n = h_points.size();
  clue::Clusterer algo(queue, dim, dc, rhoc, dm);

  // (1) host points, library staging
  algo.make_clusters(queue, h_points);
  CHECK(h_points.clustered());
  const std::vector<int> ref(h_points.clusterIndexes().begin(), h_points.clusterIndexes().end());
  const auto info = algo.lastRunInfo();
  // (2) no queue
  std::fill(h_points.clusterIndexes().begin(), h_points.clusterIndexes().end(), -7);
  algo.make_clusters(h_points);
  CHECK(std::ranges::equal(h_points.clusterIndexes(), ref));
  // (3) host + device points
  clue::PointsDevice d_points{device, dim, n};
  std::fill(h_points.clusterIndexes().begin(), h_points.clusterIndexes().end(), -7);
  algo.make_clusters(queue, h_points, d_points);
  CHECK(std::ranges::equal(h_points.clusterIndexes(), ref));
  CHECK(d_points.clustered() && d_points.n_clusters() == (std::size_t)info.n_clusters);
  CHECK(h_points.n_clusters() == (std::size_t)info.n_clusters);
  // (4) device points only
  clue::copyToDevice(queue, d_points, h_points);
  algo.make_clusters(queue, d_points);
  auto back = clue::copyToHost(queue, d_points);
  CHECK(back.clustered() && std::ranges::equal(back.clusterIndexes(), ref));
  // (5) host points with one buffer per coordinate (gathered by the library path)
  {
    std::vector<float> x(h_points.coords(0).begin(), h_points.coords(0).end());
    std::vector<float> y(h_points.coords(1).begin(), h_points.coords(1).end());
    std::vector<float> w(h_points.weights().begin(), h_points.weights().end());
    std::vector<int> ids(n, -7);
    clue::PointsHost split(dim, n, x.data(), y.data(), w.data(), ids.data());
    algo.make_clusters(queue, split);
    CHECK(std::ranges::equal(ids, ref));
  }
  // (6) device points over caller device buffers, one per coordinate
  {
    void *dx = nullptr, *dy = nullptr, *dw = nullptr, *di = nullptr;
    const std::size_t b = (std::size_t)n * 4;
    clue::detail::check(clue_device_alloc(0, b, &dx));
    clue::detail::check(clue_device_alloc(0, b, &dy));
    clue::detail::check(clue_device_alloc(0, b, &dw));
    clue::detail::check(clue_device_alloc(0, b, &di));
    clue_memcpy_htod(dx, h_points.view().coords[0], b, nullptr);
    clue_memcpy_htod(dy, h_points.view().coords[1], b, nullptr);
    clue_memcpy_htod(dw, h_points.view().weight, b, nullptr);
    clue::PointsDevice ext(device, dim, n, (float*)dx, (float*)dy, (float*)dw, (int*)di);
    algo.make_clusters(queue, ext);
    CHECK(to_host<int>(ext.clusterIndexes()) == ref);
    clue_device_free(dx);
    clue_device_free(dy);
    clue_device_free(dw);
    clue_device_free(di);
  }
  // association maps: host and device agree
  auto hmap = algo.getClusters(h_points);
  auto dmap = algo.getClusters(queue, d_points);
  auto dmap_h = dmap.toHost(queue);
  CHECK(hmap.size() == dmap.size() && hmap.size() == (std::size_t)info.n_clusters);
  CHECK(std::ranges::equal(hmap.extract().keys, dmap_h.extract().keys));
  CHECK(std::ranges::equal(hmap.extract().values, dmap_h.extract().values));
  CHECK(h_points.cluster_sizes().size() == hmap.size());

  // outputs for the oracle comparison
  const auto is_seed = to_host<int>(d_points.isSeed());
  const auto nh = to_host<int>(d_points.nearestHigher());
  const auto rho = to_host<float>(d_points.rho());
  const auto delta = to_host<float>(d_points.delta());
  std::ofstream f(out);
  f.precision(9);
  f << "x0,x1,weight,cluster_id,is_seed,nearest_higher,rho_bits,delta_bits\n";
  for (int i = 0; i < n; ++i)
    f << h_points.coords(0)[i] << "," << h_points.coords(1)[i] << "," << h_points.weights()[i] << "," << ref[i] << ","
      << is_seed[i] << "," << nh[i] << "," << bits(rho[i]) << "," << bits(delta[i]) << "\n";
  f.close();
  // silhouette on the GPU equals the host evaluation bit for bit
  const float sil = clue::silhouette(h_points);
  const float sil_dev = clue::silhouette(queue, d_points);
  CHECK(bits(sil) == bits(sil_dev));
  // centroids on the GPU equal the host evaluation bit for bit
  const auto cen_host = clue::cluster_centroids(h_points);
  const auto cen_dev = clue::cluster_centroids(queue, d_points);
  CHECK(cen_host.size() == cen_dev.size() && cen_dev.size() == (std::size_t)info.n_clusters);
  for (std::size_t c = 0; c < cen_host.size() && c < cen_dev.size(); ++c)
    for (std::size_t d = 0; d < 2; ++d) CHECK(bits(cen_host[c][d]) == bits(cen_dev[c][d]));
  CHECK(clue::validate_results(back, h_points));
  std::printf("silhouette=%.6f n_clusters=%lld dropped=%lld\n", sil, (long long)info.n_clusters,
              (long long)info.dropped_seeds);
  return 0;
}

int main(int argc, char** argv) {
  if (argc >= 3 && std::string(argv[1]) == "cpu") {
    test_kernels();
    test_metrics();
    test_host_points();
    test_association_map();
    test_properties_io(argv[2]);
  } else if (argc >= 7 && std::string(argv[1]) == "gpu") {
    try {
      run_gpu(argv[2], std::stof(argv[3]), std::stof(argv[4]), std::stof(argv[5]), argv[6]);
    } catch (const std::exception& e) {
      std::fprintf(stderr, "FAIL exception: %s\n", e.what());
      ++g_failures;
    }
  } else {
    std::fprintf(stderr, "usage: test_api cpu <dir> | gpu <in.csv> <dc> <rhoc> <dm> <out.csv>\n");
    return 2;
  }
  std::printf("%s (%d failures)\n", g_failures ? "FAILED" : "PASSED", g_failures);
  return g_failures ? 1 : 0;
}
