// Minimal TNL::Containers::Array / ArrayView stand-in (host memory only), written for
// this project so that the reference headers compile with g++.  Only the members the
// reference's hot-path headers call are provided: constructors (size, size+value,
// initializer list), cross-device assignment, setSize/resize/setValue, getSize,
// getView/getConstView, getElement/setElement, operator[] and operator().
//
// Oracle-only test infrastructure.
#pragma once
#include <cstddef>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <type_traits>

#include <TNL/Devices/Devices.h>

namespace TNL {
namespace Containers {

template <typename T, typename Device = Devices::Host, typename Index = int>
class ArrayView {
 public:
  using ValueType = T;
  using IndexType = Index;
  ArrayView() = default;
  ArrayView(T* data, Index size) : data_(data), size_(size) {}
  template <typename U, typename = std::enable_if_t<std::is_same_v<const U, T>>>
  ArrayView(const ArrayView<U, Device, Index>& v) : data_(v.getData()), size_(v.getSize()) {}

  T& operator[](Index i) const { return data_[i]; }
  T& operator()(Index i) const { return data_[i]; }
  T getElement(Index i) const { return data_[i]; }
  void setElement(Index i, const T& v) const { data_[i] = v; }
  Index getSize() const { return size_; }
  T* getData() const { return data_; }
  ArrayView getView() const { return *this; }
  ArrayView<const std::remove_const_t<T>, Device, Index> getConstView() const {
    return ArrayView<const std::remove_const_t<T>, Device, Index>(data_, size_);
  }

 private:
  T* data_ = nullptr;
  Index size_ = 0;
};

template <typename T, typename Device = Devices::Host, typename Index = int>
class Array {
 public:
  using ValueType = T;
  using IndexType = Index;
  using ViewType = ArrayView<T, Device, Index>;
  using ConstViewType = ArrayView<const T, Device, Index>;

  Array() = default;
  explicit Array(Index n) { setSize(n); }
  Array(Index n, const T& value) {
    setSize(n);
    setValue(value);
  }
  Array(std::initializer_list<T> list) {
    setSize(static_cast<Index>(list.size()));
    Index i = 0;
    for (const T& v : list) data_[i++] = v;
  }
  Array(const Array& other) { assign(other.data_.get(), other.size_); }
  Array(Array&&) noexcept = default;
  template <typename OtherDevice>
  Array(const Array<T, OtherDevice, Index>& other) {
    assign(other.getData(), other.getSize());
  }
  Array& operator=(const Array& other) {
    if (this != &other) assign(other.data_.get(), other.size_);
    return *this;
  }
  Array& operator=(Array&&) noexcept = default;
  template <typename OtherDevice>
  Array& operator=(const Array<T, OtherDevice, Index>& other) {
    assign(other.getData(), other.getSize());
    return *this;
  }

  void setSize(Index n) {
    if (n == size_) return;
    data_.reset(n > 0 ? new T[n]() : nullptr);
    size_ = n;
  }
  void resize(Index n) {
    std::unique_ptr<T[]> fresh(n > 0 ? new T[n]() : nullptr);
    const Index keep = n < size_ ? n : size_;
    for (Index i = 0; i < keep; ++i) fresh[i] = data_[i];
    data_ = std::move(fresh);
    size_ = n;
  }
  void resize(Index n, const T& value) {
    const Index old = size_;
    resize(n);
    for (Index i = old; i < n; ++i) data_[i] = value;
  }
  void setValue(const T& v) {
    for (Index i = 0; i < size_; ++i) data_[i] = v;
  }
  Index getSize() const { return size_; }
  T* getData() const { return data_.get(); }
  T getElement(Index i) const { return data_[i]; }
  void setElement(Index i, const T& v) { data_[i] = v; }
  T& operator[](Index i) { return data_[i]; }
  const T& operator[](Index i) const { return data_[i]; }
  T& operator()(Index i) { return data_[i]; }
  const T& operator()(Index i) const { return data_[i]; }
  ViewType getView() const { return ViewType(data_.get(), size_); }
  ConstViewType getConstView() const { return ConstViewType(data_.get(), size_); }

 private:
  void assign(const T* src, Index n) {
    setSize(n);
    for (Index i = 0; i < n; ++i) data_[i] = src[i];
  }
  std::unique_ptr<T[]> data_;
  Index size_ = 0;
};

}  // namespace Containers
}  // namespace TNL
