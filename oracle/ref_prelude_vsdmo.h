/* Forced-include prelude for compiling the reference's mesh and DMO translation units
 * (VSDMO/src/mesh/*.cu, VSDMO/src/dmo/*.cu, dmo/surfaceP/*.cu) unmodified with nvcc 12.9 on
 * Linux. TEST INFRASTRUCTURE ONLY: the result, oracle/_ref/libref_vsdmo.so, is the reference run
 * as a checker; nothing in the library includes this file or links that object.
 *
 * The sources were written against MSVC and an older Thrust. Three gaps keep them from building
 * as they lie; each is bridged here, in a header of our own, without changing a reference line:
 *   1. standard headers that MSVC brings in transitively (<cmath>, <sstream>, <thrust/remove.h>,
 *      ...), and std::sqrtf (ref_prelude.h);
 *   2. thrust::tuple<...>::get<N>() members: CCCL 12.9's thrust::tuple is an alias of
 *      cuda::std::tuple, which has none (mesh/MeshGPUCommon.h:128-136 calls them). The name
 *      `thrust` is mapped to a namespace that re-exports all of Thrust and adds a tuple with the
 *      member (plus the tuple_size / tuple_element traits and a zip_iterator that unwraps it);
 *   3. comparators whose operator() takes non-const references (triangleSort, quadSort,
 *      mesh/MeshGPUCommon.h:13-61), which CUB's merge sort calls with const values: the mapped
 *      thrust::sort(first, last, cmp) hands the comparator copies.
 * Every Thrust header the reference includes is included here first, before the mapping, so
 * Thrust itself is compiled as shipped. */
#pragma once
#include "ref_prelude.h"

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusparse.h>
#include <cub/cub.cuh>
#include <thrust/binary_search.h>
#include <thrust/copy.h>
#include <thrust/count.h>
#include <thrust/device_allocator.h>
#include <thrust/device_free.h>
#include <thrust/device_malloc.h>
#include <thrust/device_ptr.h>
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/extrema.h>
#include <thrust/fill.h>
#include <thrust/find.h>
#include <thrust/for_each.h>
#include <thrust/functional.h>
#include <thrust/gather.h>
#include <thrust/host_vector.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/permutation_iterator.h>
#include <thrust/iterator/transform_iterator.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/partition.h>
#include <thrust/reduce.h>
#include <thrust/remove.h>
#include <thrust/replace.h>
#include <thrust/scan.h>
#include <thrust/scatter.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/tuple.h>
#include <thrust/unique.h>
#include <array>
#include <chrono>
#include <fstream>
#include <map>
#include <numeric>
#include <set>
#include <sstream>
#include <unordered_map>
#include <utility>

namespace vsdmo_ref_thrust {
using namespace ::thrust;

template <class... T>
struct tuple : ::cuda::std::tuple<T...> {
    using base = ::cuda::std::tuple<T...>;
    using base::base;
    __host__ __device__ tuple(const base& b) : base(b) {}
    template <class U, class = ::cuda::std::enable_if_t<!::cuda::std::is_same<::cuda::std::decay_t<U>, base>::value &&
                                                         ::cuda::std::is_constructible<base, const U&>::value>>
    __host__ __device__ tuple(const U& u) : base(u) {}
    template <int N>
    __host__ __device__ const auto& get() const { return ::cuda::std::get<N>(static_cast<const base&>(*this)); }
};

template <class T> struct unwrap_tuple { using type = T; };
template <class... T> struct unwrap_tuple<tuple<T...>> { using type = ::cuda::std::tuple<T...>; };
template <class T> using zip_iterator = ::thrust::zip_iterator<typename unwrap_tuple<T>::type>;

template <class Cmp>
struct by_value_compare {
    mutable Cmp cmp;
    template <class A, class B>
    __host__ __device__ bool operator()(const A& a, const B& b) const {
        A x = a;
        B y = b;
        return cmp(x, y);
    }
};
template <class It, class Cmp>
void sort(It first, It last, Cmp cmp) { ::thrust::sort(first, last, by_value_compare<Cmp>{cmp}); }
}  // namespace vsdmo_ref_thrust

_LIBCUDACXX_BEGIN_NAMESPACE_STD
template <class... T>
struct tuple_size<vsdmo_ref_thrust::tuple<T...>> : tuple_size<tuple<T...>> {};
template <size_t I, class... T>
struct tuple_element<I, vsdmo_ref_thrust::tuple<T...>> : tuple_element<I, tuple<T...>> {};
_LIBCUDACXX_END_NAMESPACE_STD

#define thrust vsdmo_ref_thrust
