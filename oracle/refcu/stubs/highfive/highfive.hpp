// highfive/highfive.hpp (stub) -- TEST INFRASTRUCTURE ONLY (HighFive and
// HDF5 are not installed here).  The
// reference's Grid::store writes HDF5 files through HighFive; the checker
// never calls it, so only the names it uses are declared.
#pragma once
namespace HighFive {
struct DataSpace {
    template <class D> explicit DataSpace(const D &) {}
};
struct DataSet {
    template <class P> void write_raw(P) {}
};
struct File {
    enum { Truncate = 1 };
    File(const char *, int) {}
    template <class T> DataSet createDataSet(const char *, const DataSpace &) { return {}; }
};
}  // namespace HighFive
