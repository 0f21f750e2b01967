// Minimal TNL::Containers::NDArray stand-in for 2-D and 3-D row-major arrays
// (SizesHolder<Index,0,0[,0]>, std::index_sequence<0,1[,2]>): element (i,j) lives at
// i*size1 + j, so fArray(direction, cell) is the structure-of-arrays layout [27][N] the
// reference allocates with setSizes(27, N).
//
// Oracle-only test infrastructure.
#pragma once
#include <array>
#include <cstddef>
#include <utility>

#include <TNL/Containers/Array.h>

namespace TNL {
namespace Containers {

template <typename Index, Index... Sizes>
struct SizesHolder {
  static constexpr std::size_t dimension = sizeof...(Sizes);
};

namespace shim_detail {
template <typename T, typename Index, std::size_t Dim>
struct NDView {
  T* data = nullptr;
  std::array<Index, Dim> sizes{};
  template <typename... I>
  T& operator()(I... idx) const {
    static_assert(sizeof...(I) == Dim, "index count");
    const Index ids[Dim] = {static_cast<Index>(idx)...};
    Index off = 0;
    for (std::size_t d = 0; d < Dim; ++d) off = off * sizes[d] + ids[d];
    return data[off];
  }
  template <typename... I>
  T getElement(I... idx) const {
    return (*this)(idx...);
  }
  template <typename... I>
  void setElement(T v, I... idx) const {
    (*this)(idx...) = v;
  }
  NDView getView() const { return *this; }
  NDView<const std::remove_const_t<T>, Index, Dim> getConstView() const {
    return {data, sizes};
  }
};
}  // namespace shim_detail

template <typename T, typename SizesHolderT, typename Permutation, typename Device = Devices::Host>
class NDArray;

template <typename T, typename Index, Index... Sizes, std::size_t... Perm, typename Device>
class NDArray<T, SizesHolder<Index, Sizes...>, std::index_sequence<Perm...>, Device> {
  static constexpr std::size_t Dim = sizeof...(Sizes);

 public:
  using ViewType = shim_detail::NDView<T, Index, Dim>;
  using ConstViewType = shim_detail::NDView<const T, Index, Dim>;

  NDArray() = default;
  NDArray(const NDArray&) = default;
  NDArray& operator=(const NDArray&) = default;
  template <typename OtherDevice>
  NDArray& operator=(const NDArray<T, SizesHolder<Index, Sizes...>, std::index_sequence<Perm...>,
                                   OtherDevice>& other) {
    sizes_ = other.getSizesArray();
    storage_ = other.getStorageArray();
    return *this;
  }

  template <typename... S>
  void setSizes(S... s) {
    static_assert(sizeof...(S) == Dim, "size count");
    sizes_ = {static_cast<Index>(s)...};
    Index total = 1;
    for (Index v : sizes_) total *= v;
    storage_.setSize(total);
  }
  template <std::size_t D>
  Index getSize() const {
    return sizes_[D];
  }
  Index getStorageSize() const { return storage_.getSize(); }
  const std::array<Index, Dim>& getSizesArray() const { return sizes_; }
  const Array<T, Device, Index>& getStorageArray() const { return storage_; }
  Array<T, Device, Index>& getStorageArray() { return storage_; }
  void setValue(const T& v) { storage_.setValue(v); }
  T* getData() const { return storage_.getData(); }

  template <typename... I>
  T& operator()(I... idx) {
    return getView()(idx...);
  }
  template <typename... I>
  T getElement(I... idx) const {
    return getConstView()(idx...);
  }
  ViewType getView() const { return ViewType{storage_.getData(), sizes_}; }
  ConstViewType getConstView() const { return ConstViewType{storage_.getData(), sizes_}; }

 private:
  std::array<Index, Dim> sizes_{};
  Array<T, Device, Index> storage_;
};

}  // namespace Containers
}  // namespace TNL
