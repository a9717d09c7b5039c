// Link-time output shim for the compiled reference (test infrastructure only).
//
// The reference writes every result file (Temperature.dat, TempLattice.dat,
// HeatFlux.dat, Tempband.dat; src/StaticBTESynthetic/StaticBTESynthetic.cpp:
// 2613-2653, src/Solution/Solution.cpp:128-146) through std::ostream with the
// stream default of 6 significant digits, which is too coarse to check parity
// at 1e-9. This file defines the out-of-line member that every
// `stream << double` in those sources calls (std::ostream::_M_insert<double>),
// so that the statically linked definition here is used instead of the one in
// libstdc++.so: doubles are printed with 17 significant digits (they
// round-trip). When a field width is set (the setw(15) columns of
// HeatFlux.dat), a separating blank is always emitted so long numbers cannot
// run together. No reference source line is changed.
#include <locale>
#include <ostream>
#include <sstream>
#include <string>

std::ostream &gbte_ref_insert_double(std::ostream *os, double v) __asm__("_ZNSo9_M_insertIdEERSoT_");

std::ostream &gbte_ref_insert_double(std::ostream *os, double v) {
    std::ostringstream tmp;
    tmp.imbue(os->getloc());
    tmp.flags(os->flags());
    tmp.precision(17);
    tmp << static_cast<long double>(v);  // long double path: no recursion into this shim
    std::string s = tmp.str();
    std::streamsize w = os->width();
    os->width(0);
    if (w > 0) {
        s = " " + s;
        if (static_cast<std::streamsize>(s.size()) < w) s = std::string(w - s.size(), os->fill()) + s;
    }
    os->write(s.data(), static_cast<std::streamsize>(s.size()));
    return *os;
}
