// Test stand-in for LAMMPS's Memory (create / destroy of 1D and 2D arrays).
#ifndef STUB_MEMORY_H
#define STUB_MEMORY_H
namespace LAMMPS_NS {
class Memory {
 public:
  template <typename T> T *create(T *&a, int n, const char *) { a = new T[n > 0 ? n : 1](); return a; }
  template <typename T> T **create(T **&a, int n1, int n2, const char *) {
    T *data = new T[(n1 > 0 ? n1 : 1) * (n2 > 0 ? n2 : 1)]();
    a = new T *[n1 > 0 ? n1 : 1];
    for (int i = 0; i < n1; ++i) a[i] = data + (long) i * n2;
    return a;
  }
  template <typename T> void destroy(T *&a) { delete[] a; a = nullptr; }
  template <typename T> void destroy(T **&a) {
    if (a) delete[] a[0];
    delete[] a;
    a = nullptr;
  }
};
}  // namespace LAMMPS_NS
#endif
