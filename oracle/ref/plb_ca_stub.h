/*
 * plb_ca_stub.h -- the Palabos lattice surface that the reference's
 * cellular-automaton processors touch, so that pushExcessBiomass3D,
 * halfPushExcessBiomass3D (src/complab3d_processors_part1.hh:433-894),
 * updateLocalMaskNtotalLattices3D and updateAgeDistance3D
 * (src/complab3d_processors_part2.hh:71-212, 717-830) can be instantiated and
 * run on one block.  Test infrastructure: used only to build oracle/_ref.
 *
 * A lattice is one block of nx x ny x nz D3Q7 cells with a one-cell envelope
 * on every side (Palabos's default envelope width); the block sits at the
 * origin, so relative displacements and the location are zero.  A cell holds
 * seven populations and the omega of its dynamics; its density is
 * 1 + sum of the populations, the advection-diffusion convention in which
 * the reference writes a scalar d as (d-1)/4, (d-1)/8 x 6.
 */
#ifndef PLB_CA_STUB_H
#define PLB_CA_STUB_H
#include "plb_stub.h"
#include <cstdint>

namespace plb {
namespace modif { const ModifT allVariables = dataStructure; }

template<typename T, template<typename U> class D>
class BlockLattice3D {
public:
    struct Dynamics {
        T omega = 0;
        void setOmega(T w) { omega = w; }
        T getOmega() const { return omega; }
    };
    struct Cell {
        Array<T, 7> f;
        Dynamics dyn;
        Cell() { for (int i = 0; i < 7; ++i) f.d[i] = 0; }
        T computeDensity() const {
            T rhoBar = f.d[0];
            for (int i = 1; i < 7; ++i) rhoBar += f.d[i];
            return rhoBar + (T)1;
        }
        void getPopulations(Array<T, 7>& g) const { g = f; }
        void setPopulations(const Array<T, 7>& g) { f = g; }
        Dynamics& getDynamics() { return dyn; }
    };
    BlockLattice3D(plint nx_, plint ny_, plint nz_)
        : nx(nx_), ny(ny_), nz(nz_), cells((size_t)(nx_ + 2) * (ny_ + 2) * (nz_ + 2)) {}
    Cell& get(plint x, plint y, plint z) {
        return cells[((size_t)(x + 1) * (ny + 2) + (size_t)(y + 1)) * (nz + 2) + (size_t)(z + 1)];
    }
    Dot3D getLocation() const { return Dot3D{0, 0, 0}; }
    // the scalar d written as the reference writes it
    void setScalar(plint x, plint y, plint z, T d) {
        Array<T, 7> g;
        g[0] = (T)(d - 1) / 4;
        for (int i = 1; i < 7; ++i) g[i] = (T)(d - 1) / 8;
        get(x, y, z).setPopulations(g);
    }
    plint nx, ny, nz;
private:
    std::vector<Cell> cells;
};

template<typename T, template<typename U> class D>
using Cell = typename BlockLattice3D<T, D>::Cell;

template<typename T, template<typename U> class D>
Dot3D computeRelativeDisplacement(const BlockLattice3D<T, D>&, const BlockLattice3D<T, D>&) { return Dot3D{0, 0, 0}; }
}  // namespace plb

template<typename U> struct CaStubD3Q7 {};

#endif
