// No-op replacement for ValidityChecker::write_debug_info, linked in with
// ld --wrap to time the reference without its per-stage text dump of the whole
// primitive field (Solver.cpp:66 -> SolverData.cpp:203-221).
// ORACLE-ONLY TEST INFRASTRUCTURE (CPU-baseline variant).
// The member function takes (this, const VecField&, std::string by value); the
// Itanium C++ ABI passes the string by invisible reference and the caller
// destroys it, so an empty function with three pointer arguments is enough.
extern "C" void __wrap__ZNK15ValidityChecker16write_debug_infoERK8VecFieldNSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEE(
    const void*, const void*, void*) {}
