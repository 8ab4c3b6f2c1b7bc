// Driver contract of the reference (CommonFiles/Permanent.h:36-91): a
// Permanent owns its matrix (and deletes it), computePermanent() prepares the
// matrix and calls the virtual permanentFunction().  Drivers that want a
// sparse layout override prepare() (the reference keys this on a global flag
// set by the algorithm selector, Permanent.h:82-87; here the driver type
// carries it, so concurrent computations do not share state).
#pragma once

#include "Matrix.h"
#include "Settings.h"

template <class C, class S>
class Permanent {
public:
    Permanent(Matrix<S>* matrix, Settings settings) : m_Matrix(matrix), m_Settings(settings) {}
    Permanent(const Permanent&) = delete;
    Permanent& operator=(const Permanent&) = delete;
    Permanent(Permanent&&) = delete;
    Permanent& operator=(Permanent&&) = delete;
    virtual ~Permanent() { delete m_Matrix; }

    double computePermanent()
    {
        prepare();
        return permanentFunction();
    }
    virtual double permanentFunction() = 0;

    Matrix<S>* m_Matrix;
    Settings m_Settings;

protected:
    virtual void prepare() {}
};
