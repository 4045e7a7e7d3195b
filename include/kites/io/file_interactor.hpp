// file_interactor.hpp -- open a file or throw (farkhor/KiTES
// kites/io/file_interactor.hpp:15-20).
#ifndef KITES_B200_FILE_INTERACTOR_HPP_
#define KITES_B200_FILE_INTERACTOR_HPP_

#include <fstream>
#include <stdexcept>
#include <string>

namespace kites {
namespace io {

template <typename T_file>
void openFileToAccess(T_file &f, const std::string &name) {
  f.open(name.c_str());
  if (!f) throw std::runtime_error("Failed to open specified file: " + name + "\n");
}

}  // namespace io
}  // namespace kites

#endif
