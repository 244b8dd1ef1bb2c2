// C++-linkage aliases of the reference-compatible entry points.
//
// The reference programs declare their host functions with C++ linkage
// (PEGen_RayTracing_CircularHole/PESysMatGen.h:4-5, ScatterGen_*/scatter.h:4-5), so their
// unmodified main() objects reference the mangled symbols.  Exporting these aliases from
// libsysmat.so lets those objects link against this library unchanged.  This translation
// unit does not include sysmat.h: there the same names are declared with C linkage.
extern "C" {
int sysmat_legacy_pe(float*, float*, float*, float*, int);
int sysmat_legacy_scatter(float*, float*, float*, float*, float*, const char*, const char*, float*, int);
int sysmat_legacy_scatter_collimator(float*, float*, float*, float*, float*, const char*, float*, int);
int sysmat_legacy_scatter_crystal(float*, float*, float*, float*, const char*, float*, int);
}

#define SYSMAT_CXX_API __attribute__((visibility("default")))

SYSMAT_CXX_API int PESysMatGen(float* pC, float* pD, float* pI, float* dst, int cuda_id)
{
    return sysmat_legacy_pe(pC, pD, pI, dst, cuda_id);
}

SYSMAT_CXX_API int scatter(float* pC, float* pD, float* pI, float* pP, float* pe, const char* geo_crystal,
                           const char* geo_collimator, float* dst, int cuda_id)
{
    return sysmat_legacy_scatter(pC, pD, pI, pP, pe, geo_crystal, geo_collimator, dst, cuda_id);
}

SYSMAT_CXX_API int scatter(float* pC, float* pD, float* pI, float* pP, float* pe, const char* geo,
                           float* dst, int cuda_id)
{
    return sysmat_legacy_scatter_collimator(pC, pD, pI, pP, pe, geo, dst, cuda_id);
}

SYSMAT_CXX_API int scatter(float* pD, float* pI, float* pP, float* pe, const char* geo, float* dst,
                           int cuda_id)
{
    return sysmat_legacy_scatter_crystal(pD, pI, pP, pe, geo, dst, cuda_id);
}
