// G4ThreeVector.hh stand-in for tests that compile the reference's own
// Geant4-free headers (include/g4go/optical/Scene.hpp, PhotonTransport.hpp)
// and src/optical/Scene.cpp without CLHEP. TEST INFRASTRUCTURE ONLY.
//
// Those files use a three-vector of doubles with x(), y(), z() and brace
// construction; this class gives that, plus the arithmetic a test's scene
// builder needs. It is written from CLHEP's documented Hep3Vector interface,
// not copied from it.
#pragma once

#include <cmath>

class G4ThreeVector {
public:
    G4ThreeVector() = default;
    G4ThreeVector(double x, double y, double z) : fX{x}, fY{y}, fZ{z} {}

    double x() const { return fX; }
    double y() const { return fY; }
    double z() const { return fZ; }
    double dot(const G4ThreeVector& v) const { return fX * v.fX + fY * v.fY + fZ * v.fZ; }
    double mag2() const { return dot(*this); }
    double mag() const { return std::sqrt(mag2()); }
    G4ThreeVector cross(const G4ThreeVector& v) const {
        return {fY * v.fZ - fZ * v.fY, fZ * v.fX - fX * v.fZ, fX * v.fY - fY * v.fX};
    }
    G4ThreeVector unit() const {
        const double m{mag()};
        return m > 0.0 ? G4ThreeVector{fX / m, fY / m, fZ / m} : *this;
    }
    G4ThreeVector operator+(const G4ThreeVector& v) const { return {fX + v.fX, fY + v.fY, fZ + v.fZ}; }
    G4ThreeVector operator-(const G4ThreeVector& v) const { return {fX - v.fX, fY - v.fY, fZ - v.fZ}; }
    G4ThreeVector operator*(double s) const { return {fX * s, fY * s, fZ * s}; }

private:
    double fX{};
    double fY{};
    double fZ{};
};
