/*
 * plb_stub.h -- the smallest set of Palabos declarations that lets the
 * reference's Palabos-free code (EquilibriumChemistry in
 * src/complab3d_processors_part4_eqsolver.hh, defineSurrogateModel in
 * surrogateModel.hh, the example rate-law headers) compile on its own.
 * Test infrastructure: used only to build oracle/_ref, the reference's own
 * CPU code that pins the oracle.  The processor classes in those headers are
 * templates that are never instantiated, so their Palabos base classes and
 * types only need to be declared.
 */
#ifndef PLB_STUB_H
#define PLB_STUB_H
#include <cmath>
#include <vector>
#include <string>
#include <iostream>
#include <iomanip>
#include <algorithm>
namespace plb {
typedef long long plint;
typedef unsigned long long pluint;
struct Box3D { plint x0, x1, y0, y1, z0, z1; };
struct Dot3D { plint x, y, z; };
template<typename T, int n> struct Array { T d[n]; T& operator[](plint i) { return d[i]; } };
template<typename T, template<typename U> class D> class BlockLattice3D;
template<typename T, template<typename U> class D> class LatticeBoxProcessingFunctional3D {
public: virtual ~LatticeBoxProcessingFunctional3D() {} };
namespace modif { enum ModifT { nothing, staticVariables, dynamicVariables, dataStructure }; }
namespace BlockDomain { enum DomainT { bulk, bulkAndEnvelope }; }
namespace util { inline plint roundToInt(double v) { return (plint)std::floor(v + 0.5); } }
static std::ostream& pcout = std::cout;
}
using namespace plb;
typedef double T;
const T thrd = 1e-12;
#endif
