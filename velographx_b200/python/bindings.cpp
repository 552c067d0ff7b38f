// Python module of the B200 dynamic-BFS path.
//
// Mirrors the dynamic-BFS part of the reference's python/bindings.cpp:38-52:
// UpdateBatch, Graph, IncrementalBFS (keep_alive<1,2>, .distances as a list,
// static .unreachable), from_numpy_edges, from_scipy_csr, from_arrow_columns
// and from_arrow_table, with the same argument names, defaults and
// ValueError behaviour.  Extras (array batches, device-pointer batches,
// counters) serve benchmarks and tests.  The from_* loaders bulk-load on the
// device instead of applying one add per edge, so the loaded graph is compact.
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "velographx/incremental/bfs.hpp"
#include "velographx/incremental/connected_components.hpp"
#include "velographx/incremental/sssp.hpp"
#include "velographx/io.hpp"
#include "velographx/io/binary_graph.hpp"
#include "velographx/storage/consolidation.hpp"
#include "velographx/storage/dynamic_graph.hpp"

namespace py = pybind11;
using velographx::DynamicGraph;
using velographx::IncrementalBFS;
using velographx::IncrementalComponents;
using velographx::IncrementalSSSP;
using velographx::UpdateBatch;
using velographx::VertexId;
namespace detail = velographx::detail;

namespace {

using u32_array = py::array_t<std::uint32_t, py::array::c_style | py::array::forcecast>;
using u8_array = py::array_t<std::uint8_t, py::array::c_style | py::array::forcecast>;

void load_pairs(DynamicGraph& g, const std::uint32_t* uv, std::size_t n) {
  if (n == 0) return;  // an empty load leaves version 0, like applying an empty batch
  py::gil_scoped_release release;
  detail::check(vx_graph_bulk_load(g.handle(), uv, n));
}

DynamicGraph graph_from_numpy_edges(const u32_array& edges, bool directed) {
  const auto info = edges.request();
  if (info.ndim != 2 || info.shape[1] != 2) throw std::invalid_argument("edge array must have shape (N, 2)");
  DynamicGraph graph(0, directed);
  load_pairs(graph, static_cast<const std::uint32_t*>(info.ptr), static_cast<std::size_t>(info.shape[0]));
  return graph;
}

DynamicGraph graph_from_scipy_csr(const py::object& csr, bool directed) {
  if (!py::hasattr(csr, "indptr") || !py::hasattr(csr, "indices") || !py::hasattr(csr, "shape"))
    throw std::invalid_argument("expected a SciPy CSR-like object with indptr, indices, and shape");
  const auto shape = csr.attr("shape").cast<py::tuple>();
  if (shape.size() != 2 || shape[0].cast<py::ssize_t>() != shape[1].cast<py::ssize_t>())
    throw std::invalid_argument("CSR graph matrix must be square");
  const auto vertices = static_cast<std::size_t>(shape[0].cast<py::ssize_t>());
  auto indptr = py::array_t<std::int64_t, py::array::c_style | py::array::forcecast>(csr.attr("indptr"));
  auto indices = py::array_t<std::int64_t, py::array::c_style | py::array::forcecast>(csr.attr("indices"));
  const auto p = indptr.unchecked<1>();
  const auto idx = indices.unchecked<1>();
  if (static_cast<std::size_t>(p.shape(0)) != vertices + 1) throw std::invalid_argument("invalid CSR indptr length");
  DynamicGraph graph(vertices, directed);
  std::vector<std::uint32_t> uv;
  uv.reserve(static_cast<std::size_t>(idx.shape(0)) * 2);
  for (std::size_t u = 0; u < vertices; ++u) {
    const auto begin = p(static_cast<py::ssize_t>(u)), end = p(static_cast<py::ssize_t>(u + 1));
    if (begin < 0 || end < begin || end > idx.shape(0)) throw std::invalid_argument("invalid CSR offsets");
    for (auto pos = begin; pos < end; ++pos) {
      const auto v = idx(static_cast<py::ssize_t>(pos));
      if (v < 0 || static_cast<std::size_t>(v) >= vertices)
        throw std::invalid_argument("CSR contains out-of-range vertex id");
      if (!directed && static_cast<std::size_t>(v) < u) continue;
      uv.push_back(static_cast<std::uint32_t>(u));
      uv.push_back(static_cast<std::uint32_t>(v));
    }
  }
  load_pairs(graph, uv.data(), uv.size() / 2);
  return graph;
}

py::array arrow_column_to_numpy(const py::object& column) {
  if (!py::hasattr(column, "to_numpy")) throw std::invalid_argument("expected an Arrow-like column exposing to_numpy()");
  return py::array::ensure(column.attr("to_numpy")(py::arg("zero_copy_only") = false));
}

DynamicGraph graph_from_arrow_columns(const py::object& src_column, const py::object& dst_column, bool directed) {
  auto src = u32_array(arrow_column_to_numpy(src_column));
  auto dst = u32_array(arrow_column_to_numpy(dst_column));
  const auto s = src.unchecked<1>(), d = dst.unchecked<1>();
  if (s.shape(0) != d.shape(0)) throw std::invalid_argument("Arrow source and destination columns must have equal length");
  std::vector<std::uint32_t> uv(static_cast<std::size_t>(s.shape(0)) * 2);
  for (py::ssize_t i = 0; i < s.shape(0); ++i) {
    uv[2 * i] = s(i);
    uv[2 * i + 1] = d(i);
  }
  DynamicGraph graph(0, directed);
  load_pairs(graph, uv.data(), uv.size() / 2);
  return graph;
}

DynamicGraph graph_from_arrow_table(const py::object& table, const std::string& src_name, const std::string& dst_name,
                                    bool directed) {
  if (!py::hasattr(table, "column")) throw std::invalid_argument("expected an Arrow-like table exposing column(name)");
  return graph_from_arrow_columns(table.attr("column")(src_name), table.attr("column")(dst_name), directed);
}

// Owns one multi-root BFS handle (vx_mrbfs_*).
struct MultiRoot {
  vx_mrbfs* h = nullptr;
  std::size_t k = 0;
  MultiRoot(DynamicGraph& g, const u32_array& roots) : k(static_cast<std::size_t>(roots.size())) {
    detail::check(vx_mrbfs_create(g.handle(), roots.data(), k, &h));
  }
  ~MultiRoot() { vx_mrbfs_destroy(h); }
  MultiRoot(const MultiRoot&) = delete;
  MultiRoot& operator=(const MultiRoot&) = delete;
};

struct Arrays {
  u32_array src, dst;
  u8_array add;
  std::size_t n;
  Arrays(const u32_array& s, const u32_array& d, const u8_array& a) : src(s), dst(d), add(a) {
    if (src.ndim() != 1 || dst.ndim() != 1 || add.ndim() != 1 || src.shape(0) != dst.shape(0) ||
        src.shape(0) != add.shape(0))
      throw std::invalid_argument("src, dst and add must be 1-D arrays of equal length");
    n = static_cast<std::size_t>(src.shape(0));
  }
};

}  // namespace

PYBIND11_MODULE(_velographx, m) {
  m.doc() = "VeloGraphX dynamic-BFS path on NVIDIA B200 (device-resident graph and BFS)";

  py::class_<UpdateBatch>(m, "UpdateBatch")
      .def(py::init<>())
      .def("add", &UpdateBatch::add, py::arg("u"), py::arg("v"), py::arg("timestamp") = 0)
      .def("remove", &UpdateBatch::remove, py::arg("u"), py::arg("v"), py::arg("timestamp") = 0)
      .def("__len__", [](const UpdateBatch& b) { return b.updates.size(); })
      .def("empty", &UpdateBatch::empty);

  py::class_<DynamicGraph>(m, "Graph")
      .def(py::init<std::size_t, bool>(), py::arg("vertices") = 0, py::arg("directed") = false)
      .def("add_edge", &DynamicGraph::add_edge)
      .def("remove_edge", &DynamicGraph::remove_edge)
      .def("apply", &DynamicGraph::apply)
      .def("neighbors", &DynamicGraph::neighbors)
      .def_property_readonly("version", &DynamicGraph::version)
      .def_property_readonly("vertex_count", &DynamicGraph::vertex_count)
      .def("compact", &DynamicGraph::compact)
      // extras beyond the reference module
      .def_property_readonly("directed", &DynamicGraph::directed)
      .def_property_readonly("handle", [](DynamicGraph& g) { return reinterpret_cast<std::uintptr_t>(g.handle()); })
      .def("in_neighbors", &DynamicGraph::in_neighbors)
      .def("has_edge", &DynamicGraph::has_edge)
      .def("ensure_vertex", &DynamicGraph::ensure_vertex)
      .def("compact_neighbors",
           [](const DynamicGraph& g, VertexId u) {
             auto r = g.compact_neighbors(u);
             return std::vector<VertexId>(r.begin(), r.end());
           })
      .def("compact_in_neighbors",
           [](const DynamicGraph& g, VertexId v) {
             auto r = g.compact_in_neighbors(v);
             return std::vector<VertexId>(r.begin(), r.end());
           })
      .def("base_edge_count_directed", &DynamicGraph::base_edge_count_directed)
      .def("storage_bytes", &DynamicGraph::storage_bytes)
      .def("delta_ratio", &DynamicGraph::delta_ratio)
      .def("edge_count_directed", &DynamicGraph::edge_count_directed)
      .def("delta_edge_count", &DynamicGraph::delta_edge_count)
      .def("is_compact", &DynamicGraph::is_compact)
      .def("maybe_compact", &DynamicGraph::maybe_compact, py::arg("threshold") = 0.25)
      .def("dirty_out_segment_count", &DynamicGraph::dirty_out_segment_count)
      .def("dirty_in_segment_count", &DynamicGraph::dirty_in_segment_count)
      .def("bulk_load_edges",
           [](DynamicGraph& g, const u32_array& edges) {
             const auto info = edges.request();
             if (info.ndim != 2 || info.shape[1] != 2) throw std::invalid_argument("edge array must have shape (N, 2)");
             py::gil_scoped_release release;
             detail::check(vx_graph_bulk_load(g.handle(), static_cast<const std::uint32_t*>(info.ptr),
                                              static_cast<std::size_t>(info.shape[0])));
           })
      .def("apply_arrays",
           [](DynamicGraph& g, const u32_array& s, const u32_array& d, const u8_array& a) {
             Arrays x(s, d, a);
             if (!x.n) return;
             py::gil_scoped_release release;
             detail::check(vx_graph_apply(g.handle(), x.src.data(), x.dst.data(), x.add.data(), x.n));
           })
      .def("apply_device",
           [](DynamicGraph& g, std::uintptr_t s, std::uintptr_t d, std::uintptr_t a, std::size_t n,
              std::size_t vertex_count_after) {
             detail::check(vx_graph_apply_device(g.handle(), reinterpret_cast<const std::uint32_t*>(s),
                                                 reinterpret_cast<const std::uint32_t*>(d),
                                                 reinterpret_cast<const std::uint8_t*>(a), n, vertex_count_after));
           })
      .def("reserve",
           [](DynamicGraph& g, std::size_t max_batch_ops, std::size_t total_ops) {
             detail::check(vx_graph_reserve(g.handle(), max_batch_ops, total_ops));
           },
           py::arg("max_batch_ops"), py::arg("total_ops") = 0)
      .def_property_readonly("stream",
                             [](DynamicGraph& g) {
                               void* s = nullptr;
                               detail::check(vx_graph_stream(g.handle(), &s));
                               return reinterpret_cast<std::uintptr_t>(s);
                             })
      .def("synchronize", [](DynamicGraph& g) {
        py::gil_scoped_release release;
        detail::check(vx_graph_synchronize(g.handle()));
      });

  py::class_<IncrementalBFS>(m, "IncrementalBFS")
      .def(py::init<DynamicGraph&, VertexId, double>(), py::arg("graph"), py::arg("source"),
           py::arg("deletion_fallback_fraction") = 0.35, py::keep_alive<1, 2>())
      .def_property_readonly("distances", [](const IncrementalBFS& x) { return x.distances(); })
      .def("apply", &IncrementalBFS::apply)
      .def("recompute", &IncrementalBFS::recompute)
      .def_property_readonly_static("unreachable", [](py::object) { return IncrementalBFS::unreachable; })
      // extras
      .def_property_readonly("handle", [](IncrementalBFS& x) { return reinterpret_cast<std::uintptr_t>(x.handle()); })
      .def("mark_stale", [](IncrementalBFS& x) { x.mark_stale(); })
      .def_property_readonly("reachable_count", &IncrementalBFS::reachable_count)
      .def_property_readonly("last_deletion_candidates", &IncrementalBFS::last_deletion_candidates)
      .def_property_readonly("last_affected_vertices", &IncrementalBFS::last_affected_vertices)
      .def_property_readonly("last_used_full_recompute", &IncrementalBFS::last_used_full_recompute)
      .def("distances_array",
           [](IncrementalBFS& x) {
             std::size_t n = 0;
             detail::check(vx_bfs_distances(x.handle(), nullptr, 0, &n));
             py::array_t<std::uint32_t> out(static_cast<py::ssize_t>(n));
             if (n) {
               auto* ptr = out.mutable_data();
               py::gil_scoped_release release;
               detail::check(vx_bfs_distances(x.handle(), ptr, n, &n));
             }
             return out;
           })
      .def("stats",
           [](IncrementalBFS& x) {
             vx_bfs_stats_t s{};
             detail::check(vx_bfs_stats(x.handle(), &s));
             return py::dict(py::arg("reachable_count") = s.reachable_count,
                             py::arg("last_deletion_candidates") = s.last_deletion_candidates,
                             py::arg("last_affected_vertices") = s.last_affected_vertices,
                             py::arg("last_used_full_recompute") = s.last_used_full_recompute != 0,
                             py::arg("levels") = s.levels, py::arg("readback_bytes") = s.readback_bytes);
           })
      .def("apply_arrays",
           [](IncrementalBFS& x, const u32_array& s, const u32_array& d, const u8_array& a) {
             Arrays y(s, d, a);
             py::gil_scoped_release release;
             detail::check(vx_bfs_apply(x.handle(), y.src.data(), y.dst.data(), y.add.data(), y.n));
             x.mark_stale();
           })
      .def("apply_device",
           [](IncrementalBFS& x, std::uintptr_t s, std::uintptr_t d, std::uintptr_t a, std::size_t n,
              std::size_t vertex_count_after) {
             detail::check(vx_bfs_apply_device(x.handle(), reinterpret_cast<const std::uint32_t*>(s),
                                               reinterpret_cast<const std::uint32_t*>(d),
                                               reinterpret_cast<const std::uint8_t*>(a), n, vertex_count_after));
             x.mark_stale();
           })
      .def("distances_device_ptr",
           [](IncrementalBFS& x) {
             const std::uint32_t* p = nullptr;
             std::size_t n = 0;
             detail::check(vx_bfs_distances_device(x.handle(), &p, &n));
             return py::make_tuple(reinterpret_cast<std::uintptr_t>(p), n);
           })
      .def("reached_arcs",
           [](IncrementalBFS& x) {
             std::uint64_t a = 0;
             detail::check(vx_bfs_reached_arcs(x.handle(), &a));
             return a;
           })
      .def("apply_stream",
           [](IncrementalBFS& x, const u32_array& s, const u32_array& d, const u8_array& a,
              const py::array_t<std::uint64_t, py::array::c_style | py::array::forcecast>& offsets, bool digests,
              bool stats) {
             Arrays y(s, d, a);
             if (offsets.ndim() != 1 || offsets.shape(0) < 1) throw std::invalid_argument("offsets: 1-D, >= 1 entry");
             const std::size_t nb = static_cast<std::size_t>(offsets.shape(0)) - 1;
             if (offsets.data()[nb] > y.n) throw std::invalid_argument("offsets exceed the op arrays");
             py::array_t<std::uint64_t> dg(digests ? nb : 0);
             py::array_t<std::uint32_t> st(stats ? 4 * nb : 0);
             std::uint64_t* pd = digests ? dg.mutable_data() : nullptr;
             std::uint32_t* ps = stats ? st.mutable_data() : nullptr;
             {
               py::gil_scoped_release release;
               detail::check(vx_bfs_apply_stream(x.handle(), y.src.data(), y.dst.data(), y.add.data(), offsets.data(),
                                                 nb, pd, ps));
             }
             x.mark_stale();
             if (stats) st.resize({static_cast<py::ssize_t>(nb), static_cast<py::ssize_t>(4)});
             return py::make_tuple(dg, st);
           },
           py::arg("src"), py::arg("dst"), py::arg("add"), py::arg("offsets"), py::arg("digests") = false,
           py::arg("stats") = false)
      .def("reserve_stream",
           [](IncrementalBFS& x, std::size_t ops, std::size_t batches, std::size_t max_batch_ops) {
             detail::check(vx_bfs_reserve_stream(x.handle(), ops, batches, max_batch_ops));
           },
           py::arg("ops"), py::arg("batches"), py::arg("max_batch_ops"))
      .def("set_fused", [](IncrementalBFS& x, bool fused) { detail::check(vx_bfs_set_fused(x.handle(), fused)); })
      .def(
          "autotune",
          [](IncrementalBFS& x, const u32_array& roots) {
            if (roots.ndim() != 1) throw std::invalid_argument("roots: 1-D array");
            float c[4] = {0, 0, 0, 0};
            {
              py::gil_scoped_release release;
              detail::check(vx_bfs_autotune(x.handle(), roots.data(), static_cast<std::size_t>(roots.shape(0)), c));
            }
            x.mark_stale();
            return py::dict(py::arg("alpha") = c[0], py::arg("beta") = c[1],
                            py::arg("large_row") = static_cast<std::uint32_t>(c[2]), py::arg("mean_ms") = c[3]);
          },
          py::arg("roots"))
      .def("tuning",
           [](IncrementalBFS& x) {
             float a = 0, b = 0;
             std::uint32_t l = 0;
             detail::check(vx_bfs_get_tuning(x.handle(), &a, &b, &l));
             return py::make_tuple(a, b, l);
           })
      .def("set_accounting",
           [](IncrementalBFS& x, bool on) { detail::check(vx_bfs_set_accounting(x.handle(), on ? 1 : 0)); })
      .def("accounting",
           [](IncrementalBFS& x) {
             std::uint64_t a[5] = {0, 0, 0, 0, 0};
             detail::check(vx_bfs_accounting(x.handle(), a));
             return py::dict(py::arg("arcs_scanned") = a[0], py::arg("vertices_visited") = a[1],
                             py::arg("delta_entries") = a[2], py::arg("canonical_arcs") = a[3],
                             py::arg("batches") = a[4]);
           })
      .def("set_update_blocks",
           [](IncrementalBFS& x, std::uint32_t blocks) { detail::check(vx_bfs_set_update_blocks(x.handle(), blocks)); })
      .def("set_window_pull_fraction",
           [](IncrementalBFS& x, float f) { detail::check(vx_bfs_set_window_pull_fraction(x.handle(), f)); })
      .def("set_handover",
           [](IncrementalBFS& x, float m) { detail::check(vx_bfs_set_handover(x.handle(), m)); })
      .def("window_trace",
           [](IncrementalBFS& x) {
             std::size_t n = 0;
             detail::check(vx_bfs_window_trace(x.handle(), nullptr, 0, &n));
             std::vector<std::uint64_t> t(n);
             if (n) detail::check(vx_bfs_window_trace(x.handle(), t.data(), n, &n));
             py::list out;  // (us, frontier size, pull) per level
             const std::size_t levels = n ? (n - 1) / 2 : 0;
             for (std::size_t i = 0; i < levels; ++i)
               out.append(py::make_tuple(static_cast<double>(t[2 * i + 2] - t[2 * i]) * 1e-3,
                                         t[2 * i + 1] & 0x7FFFFFFFFFFFFFFFull, (t[2 * i + 1] >> 63) != 0));
             return out;
           })
      .def("set_stream_window",
           [](IncrementalBFS& x, std::uint32_t batches) {
             detail::check(vx_bfs_set_stream_window(x.handle(), batches));
           })
      .def("digest",
           [](IncrementalBFS& x) {
             std::uint64_t d = 0;
             detail::check(vx_bfs_digest(x.handle(), &d));
             return d;
           })
      .def("phase_trace",
           [](IncrementalBFS& x) {
             std::uint64_t t[32] = {};
             std::size_t n = 0;
             detail::check(vx_bfs_phase_trace(x.handle(), t, 32, &n));
             py::list out;
             for (std::size_t i = 0; i < n && i < 32; ++i) out.append(t[i]);
             return out;
           })
      .def("level_trace",
           [](IncrementalBFS& x) {
             std::size_t n = 0;
             detail::check(vx_bfs_level_trace(x.handle(), nullptr, 0, &n));
             std::vector<std::uint64_t> t(n);
             if (n) detail::check(vx_bfs_level_trace(x.handle(), t.data(), n, &n));
             py::list out;
             const std::size_t stamps = n / 2;  // levels + closing timestamp
             for (std::size_t i = 0; i + 1 < stamps; ++i)
               out.append(py::make_tuple(static_cast<double>(t[2 * (i + 1)] - t[2 * i]) * 1e-3,
                                         t[2 * i + 1] & 0x7FFFFFFFFFFFFFFFull, (t[2 * i + 1] >> 63) != 0));
             return out;
           })
      .def("set_tuning", [](IncrementalBFS& x, float alpha, float beta, std::uint32_t large_row) {
        detail::check(vx_bfs_set_tuning(x.handle(), alpha, beta, large_row));
      }, py::arg("alpha"), py::arg("beta"), py::arg("large_row"));

  // the reference module's IncrementalComponents (python/bindings.cpp:45)
  py::class_<IncrementalComponents>(m, "IncrementalComponents")
      .def(py::init<DynamicGraph&>(), py::arg("graph"), py::keep_alive<1, 2>())
      .def("component", &IncrementalComponents::component)
      .def("apply", &IncrementalComponents::apply)
      .def_property_readonly("last_repaired_vertices", &IncrementalComponents::last_repaired_vertices)
      .def("apply_arrays",
           [](IncrementalComponents& x, const u32_array& s, const u32_array& d, const u8_array& a) {
             Arrays y(s, d, a);
             {
               py::gil_scoped_release release;
               detail::check(vx_cc_apply(x.handle(), y.src.data(), y.dst.data(), y.add.data(), y.n));
             }
             x.mark_stale();
           })
      .def("labels_array", [](IncrementalComponents& x) {
        std::size_t n = 0;
        detail::check(vx_cc_labels(x.handle(), nullptr, 0, &n));
        py::array_t<std::uint32_t> out(static_cast<py::ssize_t>(n));
        if (n) {
          auto* ptr = out.mutable_data();
          py::gil_scoped_release release;
          detail::check(vx_cc_labels(x.handle(), ptr, n, &n));
        }
        return out;
      });
  // BasicIncrementalSSSP<DynamicGraph> (include/velographx/incremental/sssp.hpp:14-69;
  // not in the reference's Python module)
  py::class_<IncrementalSSSP>(m, "IncrementalSSSP")
      .def(py::init<DynamicGraph&, VertexId>(), py::arg("graph"), py::arg("source"), py::keep_alive<1, 2>())
      .def_property_readonly("distances", [](const IncrementalSSSP& x) { return x.distances(); })
      .def("apply", &IncrementalSSSP::apply)
      .def("recompute", &IncrementalSSSP::recompute)
      .def_property_readonly_static("unreachable", [](py::object) { return IncrementalSSSP::unreachable; });
  py::class_<MultiRoot>(m, "MultiRootBFS")
      .def(py::init<DynamicGraph&, const u32_array&>(), py::arg("graph"), py::arg("roots"), py::keep_alive<1, 2>())
      .def("run", [](MultiRoot& r) { detail::check(vx_mrbfs_run(r.h)); })
      .def("set_pull_fraction", [](MultiRoot& r, float f) { detail::check(vx_mrbfs_set_pull_fraction(r.h, f)); })
      .def("distances_array",
           [](MultiRoot& r) {
             std::size_t n = 0;
             const std::uint32_t* d = nullptr;
             detail::check(vx_mrbfs_distances_device(r.h, &d, &n));
             const auto V = static_cast<py::ssize_t>(n / r.k);
             py::array_t<std::uint32_t> out({static_cast<py::ssize_t>(r.k), V});
             auto* ptr = out.mutable_data();
             {
               py::gil_scoped_release release;
               detail::check(vx_mrbfs_distances(r.h, ptr, n, &n));
             }
             return out;
           })
      .def("reached_arcs",
           [](MultiRoot& r) {
             std::uint64_t a = 0;
             detail::check(vx_mrbfs_reached_arcs(r.h, &a));
             return a;
           })
      .def("level_trace",
           [](MultiRoot& r) {
             std::size_t n = 0;
             detail::check(vx_mrbfs_level_trace(r.h, nullptr, 0, &n));
             std::vector<std::uint64_t> t(n);
             if (n) detail::check(vx_mrbfs_level_trace(r.h, t.data(), n, &n));
             py::list out;  // (us, frontier size, pull) per level
             const std::size_t levels = n ? (n - 1) / 2 : 0;
             for (std::size_t i = 0; i < levels; ++i)
               out.append(py::make_tuple(static_cast<double>(t[2 * i + 2] - t[2 * i]) * 1e-3,
                                         t[2 * i + 1] & 0x7FFFFFFFFFFFFFFFull, (t[2 * i + 1] >> 63) != 0));
             return out;
           })
      .def_property_readonly("levels", [](MultiRoot& r) {
        std::uint32_t l = 0;
        detail::check(vx_mrbfs_levels(r.h, &l));
        return l;
      });

  // files (include/velographx/io.hpp:6, include/velographx/io/binary_graph.hpp:9-20);
  // load_edge_list returns the static graph as a (compact) Graph
  m.def(
      "load_edge_list",
      [](const std::string& path, bool directed) {
        vx_graph* g = nullptr;
        {
          py::gil_scoped_release release;
          detail::check(vx_graph_load_edge_list(path.c_str(), directed ? 1 : 0, &g));
        }
        return DynamicGraph::adopt(g);
      },
      py::arg("path"), py::arg("directed") = false);
  m.def(
      "save_binary",
      [](const DynamicGraph& g, const std::string& path) {
        py::gil_scoped_release release;
        detail::check(vx_graph_save_binary(g.handle(), path.c_str()));
      },
      py::arg("graph"), py::arg("path"));
  m.def(
      "load_binary",
      [](const std::string& path, bool directed) {
        vx_graph* g = nullptr;
        {
          py::gil_scoped_release release;
          detail::check(vx_graph_load_binary(path.c_str(), directed ? 1 : 0, &g));
        }
        return DynamicGraph::adopt(g);
      },
      py::arg("path"), py::arg("directed") = false);
  // consolidate_to_csr_snapshot (include/velographx/storage/consolidation.hpp:132-163)
  m.def(
      "consolidate_to_csr_snapshot",
      [](const DynamicGraph& src) {
        auto snap = velographx::consolidate_to_csr_snapshot(src);
        py::dict d;
        d["source_storage_bytes"] = snap.source_storage_bytes;
        d["consolidated_storage_bytes"] = snap.consolidated_storage_bytes;
        d["directed_edges"] = snap.directed_edges;
        d["graph"] = py::cast(std::move(snap.graph));
        return d;
      },
      py::arg("source"));
  m.def("neighbor_scan_ns", [](const DynamicGraph& g) { return velographx::neighbor_scan_ns(g); }, py::arg("graph"));
  m.def("from_numpy_edges", &graph_from_numpy_edges, py::arg("edges"), py::arg("directed") = false);
  m.def("from_scipy_csr", &graph_from_scipy_csr, py::arg("csr"), py::arg("directed") = false);
  m.def("from_arrow_columns", &graph_from_arrow_columns, py::arg("src"), py::arg("dst"), py::arg("directed") = false);
  m.def("from_arrow_table", &graph_from_arrow_table, py::arg("table"), py::arg("src") = "src",
        py::arg("dst") = "dst", py::arg("directed") = false);
  m.def("launch_count", []() { return vx_launch_count(); });
  m.def("last_error", []() {
    char buf[1024];
    vx_last_error(buf, sizeof buf);
    return std::string(buf);
  });
}
