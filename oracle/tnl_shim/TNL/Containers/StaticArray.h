// Minimal TNL::Containers::StaticArray stand-in (fixed-size value array with brace
// initialisation and operator[]).  Oracle-only test infrastructure.
#pragma once
#include <initializer_list>

#include <TNL/Devices/Devices.h>

namespace TNL {
namespace Containers {

template <int Size, typename T>
class StaticArray {
 public:
  StaticArray() = default;
  StaticArray(std::initializer_list<T> list) {
    int i = 0;
    for (const T& v : list) {
      if (i < Size) data_[i++] = v;
    }
  }
  T& operator[](int i) { return data_[i]; }
  const T& operator[](int i) const { return data_[i]; }
  T& x() { return data_[0]; }
  T& y() { return data_[1]; }
  T& z() { return data_[2]; }
  static constexpr int getSize() { return Size; }

 private:
  T data_[Size] = {};
};

}  // namespace Containers
}  // namespace TNL
