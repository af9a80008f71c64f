/*
 * Force-included (g++ -include) when compiling the ROME reference sources
 * for the test oracle.  It works around two constructs that the original
 * icpc build accepted and g++ rejects, without editing the sources:
 *
 *  - src/array.h:170 (VolSub::init) and src/array.h:383
 *    (Aligned1dArray::operator[]) name members of a dependent base without
 *    `this->`.  Two-phase lookup in g++ then needs a visible declaration:
 *    `inHBM` resolves to a global flag (VolSub::init only forwards it to
 *    allocMemory, so behaviour is unchanged), and `_ptr` to an object whose
 *    use fails to compile if that operator[] is ever instantiated.
 *  - src/map3d_optimizer.cpp:1035 passes `false` as a `const int*`; see
 *    ref_compat_map3d.h, used for that translation unit only.
 */
#ifndef ROME_ORACLE_REF_COMPAT_H
#define ROME_ORACLE_REF_COMPAT_H
#ifdef __cplusplus
extern bool inHBM;
struct RomeOracleNoPtrElem {
    template <typename T> operator T&() const {
        static_assert(sizeof(T) == 0, "Aligned1dArray::operator[] is unusable in the g++ oracle build");
        return *(T*)nullptr;
    }
};
struct RomeOracleNoPtr {
    RomeOracleNoPtrElem operator[](long) const { return RomeOracleNoPtrElem(); }
};
extern RomeOracleNoPtr _ptr;
#endif
#endif
