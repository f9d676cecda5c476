// C++ API checks, written like CLUEstering's doctest cases. Exit code 0 when
// every CHECK holds. argv[1]: a float32 file of the 10 x 1024-point batch
// (x planes then y then weights); argv[2]: data_32768 in the same layout;
// argv[3]: output file for the cluster ids of every make_clusters overload
// (argv[3] + ".util": centroids and silhouettes of the last one).
#include <cstdio>
#include <fstream>
#include <iostream>
#include <numeric>
#include <string>
#include <vector>

#include "CLUEstering/CLUEstering.hpp"

static int failures = 0;
#define CHECK(cond)                                                        \
  do {                                                                     \
    if (!(cond)) {                                                         \
      std::cerr << "CHECK failed: " #cond " (line " << __LINE__ << ")\n"; \
      ++failures;                                                          \
    }                                                                      \
  } while (0)
#define CHECK_THROWS(expr)   \
  do {                       \
    bool thrown_ = false;    \
    try {                    \
      expr;                  \
    } catch (...) {          \
      thrown_ = true;        \
    }                        \
    CHECK(thrown_);          \
  } while (0)

static std::vector<float> read_floats(const char* path) {
  std::ifstream f(path, std::ios::binary);
  f.seekg(0, std::ios::end);
  const auto bytes = static_cast<std::size_t>(f.tellg());
  f.seekg(0);
  std::vector<float> v(bytes / 4);
  f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(bytes));
  return v;
}

int main(int argc, char** argv) {
  if (argc < 4)
    return 2;
  auto queue = clue::get_queue(0u);

  // tests/test_clusterer.cpp:46-56, tests/test_convolutional_kernels.cpp:7-24
  CHECK_THROWS(clue::Clusterer<2>(-1.f, 10.f));
  CHECK_THROWS(clue::Clusterer<2>(1.f, -10.f));
  CHECK_THROWS(clue::Clusterer<2>(queue, -1.f, 10.f));
  CHECK_THROWS(clue::FlatKernel(0.f));
  CHECK_THROWS(clue::ExponentialKernel(1.f, -1.f));
  CHECK_THROWS(clue::GaussianKernel(0.f, 1.f));

  {  // tests/test_clustering.cpp:517-567: tags override the index tie-break
    clue::Clusterer<2> algo(queue, 1.f, 0.f, 1.f);
    std::vector<float> input{0.f, 0.f, 0.f, 0.f, 1.f, 1.f};
    std::vector<int> output(2);
    auto read_back = [&](clue::PointsDevice<2>& d) {
      std::vector<int32_t> nh(2), seed(2);
      clue_memcpy_async(nh.data(), d.nearest_higher(), 8, 1, queue.stream());
      clue_memcpy_async(seed.data(), d.is_seed(), 8, 1, queue.stream());
      queue.wait();
      return std::make_pair(nh, seed);
    };
    {
      clue::PointsHost<2> h(queue, 2, input.data(), output.data());
      clue::PointsDevice<2> d(queue, 2);
      algo.make_clusters(queue, h, d);
      auto [nh, seed] = read_back(d);
      CHECK(nh[0] == 1 && nh[1] == -1 && seed[0] == 0 && seed[1] == 1);
    }
    {
      clue::PointsHost<2> h(queue, 2, input.data(), output.data());
      std::vector<std::uint32_t> tags{100, 1};
      h.set_tags(tags);
      clue::PointsDevice<2> d(queue, 2);
      algo.make_clusters(queue, h, d);
      auto [nh, seed] = read_back(d);
      CHECK(nh[1] == 0 && nh[0] == -1 && seed[1] == 0 && seed[0] == 1);
    }
  }

  {  // tests/test_mahalanobis.cpp:11-43
    clue::Clusterer<1> algo(queue, 1.f, 0.3f);
    std::vector<float> w{1.f, 1.f};
    {
      clue::PointsHost<1> p(queue, 2);
      p.coords(0)[0] = 2.f;
      p.coords(0)[1] = 4.f;
      std::copy(w.begin(), w.end(), p.weights().begin());
      algo.make_clusters(queue, p);
      CHECK(p.n_clusters() == 2);
    }
    {
      clue::PointsHost<1> p(queue, 2);
      p.coords(0)[0] = 2.f;
      p.coords(0)[1] = 4.f;
      std::copy(w.begin(), w.end(), p.weights().begin());
      std::vector<float> sigma{2.f, 2.f};
      p.set_sigma(0, std::span(sigma));
      algo.make_clusters(queue, p, clue::metrics::Mahalanobis<1>{});
      CHECK(p.n_clusters() == 1);
    }
  }

  {  // tests/test_batched_clustering.cpp:51-108
    auto data = read_floats(argv[1]);
    const int n = static_cast<int>(data.size() / 3);
    std::vector<int> ids(n);
    clue::PointsHost<2> h(queue, n, data.data(), ids.data());
    clue::PointsDevice<2> d(queue, n);
    clue::Clusterer<2> algo(queue, 1.3f, 10.f, 1.3f);
    std::vector<uint32_t> sizes(10, 1024);
    algo.make_clusters(queue, h, d, std::span<const uint32_t>(sizes));
    CHECK(h.n_clusters() == 200);
    CHECK(algo.getSampleAssociations(queue, h).size() == 10);
    CHECK(d.n_clusters() == 200);
    CHECK(algo.getSeeds().size() == 200);
  }

  {  // tests/test_clusterer.cpp:13-44: every overload on data_32768
    auto data = read_floats(argv[2]);
    const int n = static_cast<int>(data.size() / 3);
    std::ofstream out(argv[3], std::ios::binary);
    clue::Clusterer<2> algo(queue, 1.3f, 10.f, 1.3f);
    auto dump = [&](const clue::PointsHost<2>& p) {
      out.write(reinterpret_cast<const char*>(p.clusterIndexes().data()), n * 4);
    };
    {
      std::vector<int> ids(n);
      clue::PointsHost<2> h(queue, n, data.data(), ids.data());
      algo.make_clusters(queue, h);
      dump(h);
    }
    {
      std::vector<int> ids(n);
      clue::PointsHost<2> h(queue, n, data.data(), ids.data());
      algo.make_clusters(h);
      dump(h);
    }
    {
      std::vector<int> ids(n);
      clue::PointsHost<2> h(queue, n, data.data(), ids.data());
      clue::PointsDevice<2> d(queue, n);
      algo.make_clusters(queue, h, d);
      dump(h);
    }
    {
      std::vector<int> ids(n);
      clue::PointsHost<2> h(queue, n, data.data(), ids.data());
      clue::PointsDevice<2> d(queue, n);
      clue::copyToDevice(queue, d, h);
      algo.make_clusters(queue, d);
      clue::copyToHost(queue, h, d);
      dump(h);
      const auto& clusters = h.clusters();
      CHECK(clusters.size() == h.n_clusters());
      std::size_t total = 0;
      for (std::size_t k = 0; k < clusters.size(); ++k)
        total += clusters.count(static_cast<int>(k));
      CHECK(total == static_cast<std::size_t>(
                         std::count_if(ids.begin(), ids.end(), [](int c) { return c >= 0; })));
    }
    {  // separate coordinate / weight / id buffers
      std::vector<float> x(data.begin(), data.begin() + n), y(data.begin() + n, data.begin() + 2 * n),
          w(data.begin() + 2 * n, data.end());
      std::vector<int> ids(n);
      clue::PointsHost<2> h(queue, n, x.data(), y.data(), w.data(), ids.data());
      algo.make_clusters(queue, h);
      dump(h);
      // utils/cluster_centroid.hpp and utils/scores.hpp, written for the checker:
      // k, k x 2 centroids, k x 2 weighted centroids, the mean silhouette and the
      // silhouette of the first clustered point with its index
      const auto cen = clue::cluster_centroids(h);
      const auto wcen = clue::weighted_cluster_centroids(h);
      CHECK(cen.size() == h.n_clusters() && wcen.size() == cen.size());
      CHECK(clue::cluster_centroid(h, 0) == cen[0]);
      CHECK(clue::weighted_cluster_centroid(h, cen.size()) == (clue::Centroid<2>{}));
      int first = 0;
      while (ids[first] < 0)
        ++first;
      const float sil = clue::silhouette(h);
      const float sil_first = clue::silhouette(h, static_cast<std::size_t>(first));
      std::ofstream util(std::string(argv[3]) + ".util", std::ios::binary);
      const float k = static_cast<float>(cen.size());
      util.write(reinterpret_cast<const char*>(&k), 4);
      for (const auto& c : cen)
        util.write(reinterpret_cast<const char*>(c.data()), 8);
      for (const auto& c : wcen)
        util.write(reinterpret_cast<const char*>(c.data()), 8);
      const float tail[3] = {sil, sil_first, static_cast<float>(first)};
      util.write(reinterpret_cast<const char*>(tail), 12);
    }
    {  // CUDA-graph replay and the autotuner leave the result as it is
      std::vector<int> ids(n);
      clue::PointsHost<2> h(queue, n, data.data(), ids.data());
      clue::PointsDevice<2> d(queue, n);
      clue::copyToDevice(queue, d, h);
      clue::Clusterer<2> tuned(queue, 1.3f, 10.f, 1.3f);
      tuned.autotune(queue, d, clue::EuclideanMetric<2>{}, clue::FlatKernel<>{.5f}, 1);
      tuned.set_graphs(queue, true);
      for (int r = 0; r < 2; ++r) {
        tuned.make_clusters(queue, d);
        std::vector<int> again(n);
        clue_memcpy_async(again.data(), d.clusterIndexes(), n * 4, 1, queue.stream());
        queue.wait();
        std::vector<int> plain(n);
        clue::PointsHost<2> h2(queue, n, data.data(), plain.data());
        algo.make_clusters(queue, h2);
        CHECK(again == plain);
      }
      CHECK(tuned.tuning(queue).label_jump_rounds >= -1);
    }
  }
  if (failures)
    std::cerr << failures << " check(s) failed\n";
  return failures ? 1 : 0;
}
