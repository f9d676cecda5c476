// alpaka.hpp — TEST INFRASTRUCTURE ONLY. A serial, host-only stand-in for the
// part of the alpaka API that CLUEstering's headers use, so that those headers
// compile unmodified into the reference's own serial CPU backend
// (ALPAKA_ACC_CPU_B_SEQ_T_SEQ_ENABLED) for the test suite's checker
// (oracle/ref_driver.cpp, built into oracle/_ref/). It is written from
// alpaka's documented semantics for that backend, not from alpaka's sources:
//   - one device (the host), blocking queues, no-op waits and events;
//   - buffers are reference-counted host arrays, views wrap plain pointers;
//   - a kernel launch runs the grid's blocks one after another, in row-major
//     order, with one thread per block; a thread owns `elements` consecutive
//     indices per dimension and strides by the whole grid's element count;
//   - atomics are plain read-modify-writes (nothing runs concurrently).
#pragma once

// alpaka's own header brings in much of the standard library; the reference
// headers rely on that for <numeric>, <algorithm> and friends.
#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <functional>
#include <iterator>
#include <limits>
#include <numeric>
#include <optional>
#include <ranges>
#include <span>
#include <cstdint>
#include <cstring>
#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

#ifndef ALPAKA_FN_HOST
#define ALPAKA_FN_HOST
#endif
#ifndef ALPAKA_FN_ACC
#define ALPAKA_FN_ACC
#endif
#ifndef ALPAKA_FN_HOST_ACC
#define ALPAKA_FN_HOST_ACC
#endif
#ifndef ALPAKA_FN_INLINE
#define ALPAKA_FN_INLINE inline
#endif

namespace alpaka {

// ---- dimensions and index vectors ------------------------------------------

template <std::size_t N>
using DimInt = std::integral_constant<std::size_t, N>;

template <typename TDim, typename TIdx>
struct Vec {
  static constexpr std::size_t N = TDim::value;
  std::array<TIdx, N> v{};

  constexpr Vec() = default;
  template <typename... Ts>
    requires(sizeof...(Ts) == N && N > 0 && (std::is_convertible_v<Ts, TIdx> && ...))
  constexpr Vec(Ts... xs) : v{static_cast<TIdx>(xs)...} {}

  static constexpr Vec ones() {
    Vec r;
    for (auto& x : r.v)
      x = TIdx{1};
    return r;
  }
  static constexpr Vec zeros() { return Vec{}; }
  constexpr TIdx& operator[](std::size_t i) { return v[i]; }
  constexpr const TIdx& operator[](std::size_t i) const { return v[i]; }
  constexpr TIdx prod() const {
    TIdx p{1};
    for (auto x : v)
      p *= x;
    return p;
  }
  friend constexpr Vec operator*(const Vec& a, const Vec& b) {
    Vec r;
    for (std::size_t i = 0; i < N; ++i)
      r.v[i] = a.v[i] * b.v[i];
    return r;
  }
};

template <typename T>
struct DimOf {
  using type = typename T::Dim;
};
template <typename T>
using Dim = typename DimOf<std::remove_cvref_t<T>>::type;

template <typename TDim, typename TIdx>
struct WorkDivMembers {
  using Dim = TDim;
  Vec<TDim, TIdx> blocks, threads, elems;

  WorkDivMembers(const Vec<TDim, TIdx>& b, const Vec<TDim, TIdx>& t, const Vec<TDim, TIdx>& e)
      : blocks(b), threads(t), elems(e) {}
  template <typename I>
    requires(TDim::value == 1 && std::is_integral_v<I>)
  WorkDivMembers(I b, I t, I e)
      : blocks(static_cast<TIdx>(b)), threads(static_cast<TIdx>(t)), elems(static_cast<TIdx>(e)) {}
};

// ---- origins and units of getIdx / getWorkDiv ------------------------------

struct Grid {};
struct Block {};
struct Thread {};
struct Blocks {};
struct Threads {};
struct Elems {};

// ---- platform, device, queue, event ----------------------------------------

struct DevCpu;
struct PlatformCpu {
  using Dev = DevCpu;
};
struct DevCpu {
  using Platform = PlatformCpu;
  friend bool operator==(const DevCpu&, const DevCpu&) { return true; }
  friend bool operator!=(const DevCpu&, const DevCpu&) { return false; }
  int iDevice() const { return 0; }
};
struct QueueCpuBlocking {
  using Dev = DevCpu;
  DevCpu dev;
  explicit QueueCpuBlocking(const DevCpu& d) : dev(d) {}
  friend bool operator==(const QueueCpuBlocking&, const QueueCpuBlocking&) { return true; }
};
struct QueueCpuNonBlocking : QueueCpuBlocking {
  using QueueCpuBlocking::QueueCpuBlocking;
};
struct EventCpu {
  explicit EventCpu(const DevCpu&) {}
};

template <typename T>
struct DevOf {
  using type = typename std::remove_cvref_t<T>::Dev;
};
template <typename T>
using Dev = typename DevOf<T>::type;

template <typename T>
struct PlatformOf {
  using type = typename std::remove_cvref_t<T>::Platform;
};
template <typename T>
using Platform = typename PlatformOf<T>::type;

template <typename T>
inline constexpr bool isQueue = std::is_base_of_v<QueueCpuBlocking, std::remove_cvref_t<T>>;
template <typename T>
inline constexpr bool isDevice = std::is_same_v<std::remove_cvref_t<T>, DevCpu>;
template <typename T>
inline constexpr bool isPlatform = std::is_same_v<std::remove_cvref_t<T>, PlatformCpu>;

inline DevCpu getDevByIdx(const PlatformCpu&, std::size_t) { return DevCpu{}; }
inline std::vector<DevCpu> getDevs(const PlatformCpu&) { return {DevCpu{}}; }
inline std::size_t getDevCount(const PlatformCpu&) { return 1; }
inline int getNativeHandle(const DevCpu&) { return 0; }

template <typename TQueue>
  requires isQueue<TQueue>
inline DevCpu getDev(const TQueue& q) {
  return q.dev;
}

template <typename TQueue>
  requires isQueue<TQueue>
inline void wait(const TQueue&) {}
inline void wait(const EventCpu&) {}
template <typename TQueue>
  requires isQueue<TQueue>
inline void enqueue(TQueue&, EventCpu&) {}

// ---- memory: buffers and views ---------------------------------------------

// A reference-counted host array (copies share the storage, as alpaka's
// buffers do) or a view of a plain pointer.
template <typename TDev, typename T, typename TDim, typename TIdx>
class Buf {
 public:
  using Dev = TDev;
  using Dim = TDim;
  using Elem = T;
  Buf(const TDev& dev, const Vec<TDim, TIdx>& extent)
      : m_dev(dev), m_extent(extent),
        m_store(std::make_shared<std::vector<T>>(static_cast<std::size_t>(TDim::value == 0 ? 1 : extent.prod()))) {}
  T* data() const { return m_store->data(); }
  const Vec<TDim, TIdx>& extent() const { return m_extent; }
  const TDev& dev() const { return m_dev; }
  T& operator[](std::size_t i) const { return data()[i]; }
  T& operator*() const { return *data(); }

 private:
  TDev m_dev;
  Vec<TDim, TIdx> m_extent;
  std::shared_ptr<std::vector<T>> m_store;
};

template <typename TDev, typename T, typename TDim, typename TIdx>
class ViewPlainPtr {
 public:
  using Dev = TDev;
  using Dim = TDim;
  using Elem = T;
  ViewPlainPtr(T* p, const TDev& dev, const Vec<TDim, TIdx>& extent) : m_ptr(p), m_dev(dev), m_extent(extent) {}
  T* data() const { return m_ptr; }
  const Vec<TDim, TIdx>& extent() const { return m_extent; }
  const TDev& dev() const { return m_dev; }
  T& operator[](std::size_t i) const { return m_ptr[i]; }

 private:
  T* m_ptr;
  TDev m_dev;
  Vec<TDim, TIdx> m_extent;
};

template <typename T, typename TIdx, typename TDev, typename TDim>
inline Buf<TDev, T, TDim, TIdx> allocBuf(const TDev& dev, const Vec<TDim, TIdx>& extent) {
  return Buf<TDev, T, TDim, TIdx>(dev, extent);
}
template <typename T, typename TIdx, typename TDev, typename TPlatform, typename TDim>
inline Buf<TDev, T, TDim, TIdx> allocMappedBuf(const TDev& dev, const TPlatform&, const Vec<TDim, TIdx>& extent) {
  return Buf<TDev, T, TDim, TIdx>(dev, extent);
}
template <typename T, typename TIdx, typename TQueue, typename TDim>
  requires isQueue<TQueue>
inline Buf<DevCpu, T, TDim, TIdx> allocAsyncBuf(const TQueue& q, const Vec<TDim, TIdx>& extent) {
  return Buf<DevCpu, T, TDim, TIdx>(q.dev, extent);
}

template <typename TView>
inline auto getExtents(const TView& v) {
  return v.extent();
}

template <typename TView>
inline std::size_t elem_count(const TView& v) {
  using D = typename std::remove_cvref_t<TView>::Dim;
  if constexpr (D::value == 0)
    return 1;
  else
    return static_cast<std::size_t>(v.extent().prod());
}

// Copies the destination's extent worth of elements (both views hold it).
template <typename TQueue, typename TDst, typename TSrc>
  requires isQueue<TQueue>
inline void memcpy(TQueue&, TDst&& dst, const TSrc& src) {
  const std::size_t n = std::min(elem_count(dst), elem_count(src));
  using T = typename std::remove_cvref_t<TDst>::Elem;
  if (n)
    std::memmove(static_cast<void*>(const_cast<std::remove_const_t<T>*>(dst.data())), src.data(), n * sizeof(T));
}
template <typename TQueue, typename TDst, typename TSrc, typename TExt>
  requires isQueue<TQueue>
inline void memcpy(TQueue&, TDst&& dst, const TSrc& src, const TExt& extent) {
  std::size_t n;
  if constexpr (std::is_integral_v<TExt>)
    n = static_cast<std::size_t>(extent);
  else
    n = static_cast<std::size_t>(extent.prod());
  using T = typename std::remove_cvref_t<TDst>::Elem;
  if (n)
    std::memmove(static_cast<void*>(const_cast<std::remove_const_t<T>*>(dst.data())), src.data(), n * sizeof(T));
}
template <typename TQueue, typename TView>
  requires isQueue<TQueue>
inline void memset(TQueue&, TView&& v, std::uint8_t byte) {
  using T = typename std::remove_cvref_t<TView>::Elem;
  std::memset(static_cast<void*>(const_cast<std::remove_const_t<T>*>(v.data())), byte, elem_count(v) * sizeof(T));
}
template <typename TQueue, typename TView, typename TExt>
  requires isQueue<TQueue>
inline void memset(TQueue&, TView&& v, std::uint8_t byte, const TExt& extent) {
  using T = typename std::remove_cvref_t<TView>::Elem;
  std::size_t n;
  if constexpr (std::is_integral_v<TExt>)
    n = static_cast<std::size_t>(extent);
  else
    n = static_cast<std::size_t>(extent.prod());
  std::memset(static_cast<void*>(const_cast<std::remove_const_t<T>*>(v.data())), byte, n * sizeof(T));
}
template <typename TQueue, typename TView, typename TVal>
  requires isQueue<TQueue>
inline void fill(TQueue&, TView&& v, const TVal& value) {
  auto* p = v.data();
  for (std::size_t i = 0; i < elem_count(v); ++i)
    p[i] = value;
}
template <typename TQueue, typename TView, typename TVal, typename TExt>
  requires isQueue<TQueue>
inline void fill(TQueue&, TView&& v, const TVal& value, const TExt& extent) {
  auto* p = v.data();
  std::size_t n;
  if constexpr (std::is_integral_v<TExt>)
    n = static_cast<std::size_t>(extent);
  else
    n = static_cast<std::size_t>(extent.prod());
  for (std::size_t i = 0; i < n; ++i)
    p[i] = value;
}

// ---- accelerator and kernel launch -----------------------------------------

template <typename TDim, typename TIdx>
struct AccCpuSerial {
  using Dim = TDim;
  using Idx = TIdx;
  WorkDivMembers<TDim, TIdx> wd;
  Vec<TDim, TIdx> block;  // index of the running block in the grid
};

namespace concepts {
template <typename T>
concept Acc = requires(const T& a) {
  a.wd;
  a.block;
};
}  // namespace concepts

template <typename TOrigin, typename TUnit, typename TAcc>
inline Vec<typename TAcc::Dim, typename TAcc::Idx> getIdx(const TAcc& acc) {
  using V = Vec<typename TAcc::Dim, typename TAcc::Idx>;
  if constexpr (std::is_same_v<TOrigin, Grid> && std::is_same_v<TUnit, Blocks>)
    return acc.block;
  else if constexpr (std::is_same_v<TOrigin, Block> && std::is_same_v<TUnit, Threads>)
    return V{};
  else if constexpr (std::is_same_v<TOrigin, Grid> && std::is_same_v<TUnit, Threads>)
    return acc.block * acc.wd.threads;
  else
    static_assert(sizeof(TAcc) == 0, "index origin/unit not used by the reference");
}

template <typename TOrigin, typename TUnit, typename TAcc>
inline Vec<typename TAcc::Dim, typename TAcc::Idx> getWorkDiv(const TAcc& acc) {
  if constexpr (std::is_same_v<TOrigin, Grid> && std::is_same_v<TUnit, Blocks>)
    return acc.wd.blocks;
  else if constexpr (std::is_same_v<TOrigin, Block> && std::is_same_v<TUnit, Threads>)
    return acc.wd.threads;
  else if constexpr (std::is_same_v<TOrigin, Thread> && std::is_same_v<TUnit, Elems>)
    return acc.wd.elems;
  else if constexpr (std::is_same_v<TOrigin, Block> && std::is_same_v<TUnit, Elems>)
    return acc.wd.threads * acc.wd.elems;
  else if constexpr (std::is_same_v<TOrigin, Grid> && std::is_same_v<TUnit, Threads>)
    return acc.wd.blocks * acc.wd.threads;
  else if constexpr (std::is_same_v<TOrigin, Grid> && std::is_same_v<TUnit, Elems>)
    return acc.wd.blocks * acc.wd.threads * acc.wd.elems;
  else
    static_assert(sizeof(TAcc) == 0, "work division origin/unit not used by the reference");
}

// The indices a thread owns along one dimension, below `extent`: runs of
// `elems` consecutive indices starting at (global thread index) * elems,
// stepping by the grid's element count.
template <typename TIdx>
class ElementRange {
 public:
  ElementRange(TIdx first, TIdx run, TIdx stride, TIdx extent)
      : m_first(first), m_run(run), m_stride(stride), m_extent(extent) {}
  class iterator {
   public:
    iterator(TIdx base, TIdx off, const ElementRange* r) : m_base(base), m_off(off), m_r(r) { settle(); }
    TIdx operator*() const { return m_base + m_off; }
    iterator& operator++() {
      ++m_off;
      settle();
      return *this;
    }
    bool operator!=(const iterator& o) const { return m_base != o.m_base || m_off != o.m_off; }
    bool operator==(const iterator& o) const { return !(*this != o); }

   private:
    void settle() {
      if (m_base >= m_r->m_extent) {
        m_base = m_r->end_base();
        m_off = 0;
        return;
      }
      if (m_off == m_r->m_run || m_base + m_off >= m_r->m_extent) {
        m_base += m_r->m_stride;
        m_off = 0;
        if (m_base >= m_r->m_extent) {
          m_base = m_r->end_base();
          return;
        }
      }
    }
    TIdx m_base, m_off;
    const ElementRange* m_r;
  };
  iterator begin() const { return iterator(m_first, 0, this); }
  iterator end() const { return iterator(end_base(), 0, this); }

 private:
  TIdx end_base() const { return m_extent >= m_first ? m_extent + m_run + m_stride : m_first; }
  TIdx m_first, m_run, m_stride, m_extent;
};

template <std::size_t Along, typename TAcc, typename TExt>
inline auto uniformElementsAlong(const TAcc& acc, TExt extent) {
  using TIdx = typename TAcc::Idx;
  const TIdx run = acc.wd.elems[Along];
  const TIdx thread = acc.block[Along] * acc.wd.threads[Along];
  const TIdx stride = acc.wd.blocks[Along] * acc.wd.threads[Along] * run;
  return ElementRange<TIdx>(thread * run, run, stride, static_cast<TIdx>(extent));
}
template <std::size_t Along, typename TAcc>
inline auto uniformElementsAlong(const TAcc& acc) {
  const auto grid = acc.wd.blocks[Along] * acc.wd.threads[Along] * acc.wd.elems[Along];
  return uniformElementsAlong<Along>(acc, grid);
}
template <typename TAcc, typename TExt>
  requires(TAcc::Dim::value == 1)
inline auto uniformElements(const TAcc& acc, TExt extent) {
  return uniformElementsAlong<0>(acc, extent);
}

namespace hierarchy {
struct Grids {};
struct Blocks {};
struct Threads {};
}  // namespace hierarchy

template <typename TAcc, typename T, typename TVal, typename THier = hierarchy::Grids>
  requires concepts::Acc<TAcc>
inline T atomicAdd(const TAcc&, T* p, const TVal& v, THier = THier{}) {
  const T old = *p;
  *p = static_cast<T>(old + static_cast<T>(v));
  return old;
}
template <typename TAcc, typename T, typename TVal, typename THier = hierarchy::Grids>
  requires concepts::Acc<TAcc>
inline T atomicSub(const TAcc&, T* p, const TVal& v, THier = THier{}) {
  const T old = *p;
  *p = static_cast<T>(old - static_cast<T>(v));
  return old;
}

// Runs the kernel on every block of the grid, one after another in row-major
// order (last dimension fastest), each block with its one thread.
template <typename TAcc, typename TQueue, typename TWorkDiv, typename TKernel, typename... TArgs>
  requires isQueue<TQueue>
inline void exec(TQueue&, const TWorkDiv& wd, const TKernel& kernel, TArgs&&... args) {
  using TDim = typename TAcc::Dim;
  using TIdx = typename TAcc::Idx;
  constexpr std::size_t N = TDim::value;
  WorkDivMembers<TDim, TIdx> w(wd.blocks, wd.threads, wd.elems);
  TAcc acc{w, Vec<TDim, TIdx>{}};
  std::array<TIdx, N> b{};
  const TIdx total = w.blocks.prod();
  for (TIdx k = 0; k < total; ++k) {
    TIdx rem = k;
    for (std::size_t d = N; d-- > 0;) {
      b[d] = rem % w.blocks[d];
      rem /= w.blocks[d];
    }
    acc.block.v = b;
    kernel(acc, args...);
  }
}

}  // namespace alpaka
