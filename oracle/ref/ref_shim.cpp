// Test infrastructure only: C entry points onto the reference's own host functions.
//
// The reference exports plain C++ (mangled) functions.  This shim is linked against
// the reference's unmodified .cu sources (compiled by oracle/Makefile into
// oracle/_ref/) so that tests and the reference arm of bench.py can reach them through
// ctypes.  One shared object per reference program, because the three scatter
// programs define device functions and host entry points with identical names.
//
//   PESysMatGen  PEGen_RayTracing_CircularHole/PESysMatGen.h:4-5
//   scatter      ScatterGen_RayTracing_CircularHole/scatter.h:4-5   (combined)
//   scatter      ScatterGen_Collimator/scatter.h:4-5                (collimator only)
//   scatter      ScatterGen_Crystal/scatter.h:4-5                   (crystal only)

#if defined(REF_PE)
extern int PESysMatGen(float* pC, float* pD, float* pI, float* dst, int cuda_id);
extern "C" int ref_PESysMatGen(float* pC, float* pD, float* pI, float* dst, int cuda_id)
{
    return PESysMatGen(pC, pD, pI, dst, cuda_id);
}
#elif defined(REF_SCATTER_COMBINED)
extern int scatter(float* pC, float* pD, float* pI, float* pP, float* pe, const char* geoCrystal,
                   const char* geoCollimator, float* dst, int cuda_id);
extern "C" int ref_scatter(float* pC, float* pD, float* pI, float* pP, float* pe,
                           const char* geoCrystal, const char* geoCollimator, float* dst, int cuda_id)
{
    return scatter(pC, pD, pI, pP, pe, geoCrystal, geoCollimator, dst, cuda_id);
}
#elif defined(REF_SCATTER_COLLIMATOR)
extern int scatter(float* pC, float* pD, float* pI, float* pP, float* pe, const char* geo,
                   float* dst, int cuda_id);
extern "C" int ref_scatter_collimator(float* pC, float* pD, float* pI, float* pP, float* pe,
                                      const char* geo, float* dst, int cuda_id)
{
    return scatter(pC, pD, pI, pP, pe, geo, dst, cuda_id);
}
#elif defined(REF_SCATTER_CRYSTAL)
extern int scatter(float* pD, float* pI, float* pP, float* pe, const char* geo, float* dst,
                   int cuda_id);
extern "C" int ref_scatter_crystal(float* pD, float* pI, float* pP, float* pe, const char* geo,
                                   float* dst, int cuda_id)
{
    return scatter(pD, pI, pP, pe, geo, dst, cuda_id);
}
#endif
