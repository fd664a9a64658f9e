// Host-side stand-ins for the CUDA builtins and the HOOMD-blue 2.x types that the
// reference's per-thread device functions use, so that those functions can be
// compiled unchanged for the CPU as a parity checker.
//
// This header is test infrastructure: it is only compiled by oracle/ref_recipe
// into oracle/_ref/, never linked into the product library.
//
// HOOMD-blue itself is not part of the reference checkout.  The box operations
// below restate the semantics of HOOMD 2.x BoxDim (minImage with rint on the
// device path, makeFraction, wrap with the xy tilt) for an orthorhombic box
// centred on the origin with an xy tilt only, which is all the reference uses.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <quadmath.h>

#define __global__ static
#define __device__
#define __host__
#define __forceinline__ inline
#define HOSTDEVICE

typedef float Scalar;
struct Scalar2 { float x, y; };
struct Scalar3 { float x, y, z; };
struct Scalar4 { float x, y, z, w; };
typedef Scalar2 float2_s;
typedef Scalar2 CUFFTCOMPLEX;
struct int3_s { int x, y, z; };
typedef int3_s int3;
struct dim3 { unsigned x, y, z; dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {} };

static inline Scalar2 make_scalar2(float a, float b) { return Scalar2{a, b}; }
static inline Scalar3 make_scalar3(float a, float b, float c) { return Scalar3{a, b, c}; }
static inline Scalar4 make_scalar4(float a, float b, float c, float d) { return Scalar4{a, b, c, d}; }
static inline int3 make_int3(int a, int b, int c) { return int3{a, b, c}; }

static inline Scalar3 operator+(Scalar3 a, Scalar3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline Scalar3 operator-(Scalar3 a, Scalar3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline Scalar3 operator*(Scalar s, Scalar3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline Scalar3 operator*(Scalar3 a, Scalar s) { return {s * a.x, s * a.y, s * a.z}; }
static inline Scalar3 operator/(Scalar3 a, Scalar s) { return {a.x / s, a.y / s, a.z / s}; }
static inline Scalar3 operator/(Scalar3 a, Scalar3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
static inline Scalar3 operator-(Scalar3 a) { return {-a.x, -a.y, -a.z}; }
static inline Scalar3& operator+=(Scalar3& a, Scalar3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
static inline Scalar3& operator-=(Scalar3& a, Scalar3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
static inline Scalar3& operator*=(Scalar3& a, Scalar s) { a.x *= s; a.y *= s; a.z *= s; return a; }
static inline Scalar dot(Scalar3 a, Scalar3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Thread coordinates of the emulated launch (one thread at a time).
static dim3 blockIdx, threadIdx, blockDim, gridDim;

static inline int __float2int_rd(float x) { return (int)floorf(x); }
static inline int __double2int_rd(double x) { return (int)floor(x); }
static inline float atomicAdd(float* p, float v) { float o = *p; *p = o + v; return o; }
static inline void __syncthreads() {}

// Texture fetches read straight from the bound array.
struct scalar4_tex_t {};
static scalar4_tex_t tables1_tex;
static inline Scalar4 texFetchScalar4(const Scalar4* p, scalar4_tex_t, int i) { return p[i]; }

struct BoxDim {
    Scalar3 L, lo, hi, Linv;
    Scalar xy;
    BoxDim() : BoxDim(1, 1, 1, 0) {}
    BoxDim(Scalar lx, Scalar ly, Scalar lz, Scalar xy_) {
        L = {lx, ly, lz};
        hi = {lx / 2, ly / 2, lz / 2};
        lo = {-lx / 2, -ly / 2, -lz / 2};
        Linv = {1.0f / lx, 1.0f / ly, 1.0f / lz};
        xy = xy_;
    }
    Scalar3 getL() const { return L; }
    Scalar getTiltFactorXY() const { return xy; }
    // Device-path minimum image (rint based), z then y then x.
    Scalar3 minImage(const Scalar3& v) const {
        Scalar3 w = v;
        Scalar img = rintf(w.z * Linv.z);
        w.z -= L.z * img;
        img = rintf(w.y * Linv.y);
        w.x -= L.y * xy * img;
        w.y -= L.y * img;
        w.x -= L.x * rintf(w.x * Linv.x);
        return w;
    }
    Scalar3 makeFraction(const Scalar3& v) const {
        Scalar3 d = v - lo;
        d.x -= xy * v.y;
        return d / L;
    }
    void wrap(Scalar3& w, int3& img) const {
        Scalar tilt_x = xy * w.y;
        if (w.x >= hi.x + tilt_x) { w.x -= L.x; img.x++; }
        else if (w.x < lo.x + tilt_x) { w.x += L.x; img.x--; }
        if (w.y >= hi.y) { w.y -= L.y; w.x -= L.y * xy; img.y++; }
        else if (w.y < lo.y) { w.y += L.y; w.x += L.y * xy; img.y--; }
        if (w.z >= hi.z) { w.z -= L.z; img.z++; }
        else if (w.z < lo.z) { w.z += L.z; img.z--; }
    }
};

// Minimal HOOMD array wrappers used by the setup block.
enum class access_location { host, device };
enum class access_mode { read, readwrite, overwrite };
struct ExecConf {};
template <class T> struct GPUArray {
    std::vector<T> v;
    GPUArray() {}
    GPUArray(size_t n, ExecConf*) : v(n) {}
    void swap(GPUArray& o) { v.swap(o.v); }
};
template <class T> struct ArrayHandle {
    T* data;
    ArrayHandle(GPUArray<T>& a, access_location, access_mode) : data(a.v.data()) {}
};
