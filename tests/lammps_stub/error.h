// Test stand-in for LAMMPS's Error: error->all throws, so a harness can report it.
#ifndef STUB_ERROR_H
#define STUB_ERROR_H
#include <stdexcept>
#include <string>
#define FLERR __FILE__, __LINE__
namespace LAMMPS_NS {
class Error {
 public:
  [[noreturn]] void all(const std::string &file, int line, const std::string &msg) {
    throw std::runtime_error(file + ":" + std::to_string(line) + ": " + msg);
  }
};
}  // namespace LAMMPS_NS
#endif
