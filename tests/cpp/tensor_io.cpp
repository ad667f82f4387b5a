// Exercises the tensor IO of the planc C++ API without a GPU:
//   tensor_io npy <file.npy> <out.bin>   NumPyArray::load, then Tensor::write
//   tensor_io bin <file.bin> <out.bin>   Tensor::read (.info sidecar), then Tensor::write
// and prints "modes d0 d1 ... numel sum first last" of the tensor it read.
#include <cstdio>
#include <iostream>
#include <string>

#include "planc/npyio.hpp"
#include "planc/tensor.hpp"

int main(int argc, char** argv) {
  if (argc != 4) return 2;
  const std::string how = argv[1];
  planc::Tensor t;
  if (how == "npy") {
    planc::NumPyArray a;
    a.load(argv[2]);
    t = *a.m_input_tensor;
  } else {
    t.read(argv[2]);
  }
  double s = 0;
  for (double v : t.m_data) s += v;
  std::printf("%d", t.modes());
  for (int i = 0; i < t.modes(); ++i) std::printf(" %d", t.dimension(i));
  std::printf(" %llu %.17g %.17g %.17g\n", (unsigned long long)t.numel(), s, t.m_data.front(),
              t.m_data.back());
  t.write(argv[3]);
  return 0;
}
