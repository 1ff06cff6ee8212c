// amrex_shim_core.H -- TEST INFRASTRUCTURE ONLY.
//
// A single-box, CPU-only stand-in for the part of the AMReX API that ERF's
// hot-path leaf operators use (types, index boxes, Array4 views, serial
// ParallelFor, boundary-condition records, a one-FAB MultiFab), so that those
// operators compile unmodified from the reference's own sources into
// oracle/_ref/ and pin the oracle's restatement of them.  AMReX itself (a
// git submodule of the reference) is absent; this file implements only the
// interface shapes those sources call, with serial loops.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#define AMREX_SPACEDIM 3
#define AMREX_ATTRIBUTE_WEAK __attribute__((weak))
#define AMREX_PRAGMA_SIMD
typedef double amrex_real;
#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST
#define AMREX_GPU_HOST_DEVICE
#define AMREX_FORCE_INLINE inline
#define AMREX_INLINE inline
#define AMREX_RESTRICT __restrict__
#define AMREX_D_DECL(a, b, c) a, b, c
#define AMREX_D_TERM(a, b, c) a b c
#define AMREX_ASSERT(x) ((void)0)
#define AMREX_ASSERT_WITH_MESSAGE(x, m) ((void)0)
#define AMREX_ALWAYS_ASSERT(x) do { if (!(x)) amrex::Abort("assertion failed: " #x); } while (0)
#define AMREX_ALWAYS_ASSERT_WITH_MESSAGE(x, m) do { if (!(x)) amrex::Abort(m); } while (0)
#define AMREX_GPU_ERROR_CHECK() ((void)0)
#define BL_PROFILE(x) ((void)0)
#define BL_PROFILE_VAR(x, y) ((void)0)
#define BL_PROFILE_VAR_STOP(y) ((void)0)
#define BL_PROFILE_REGION(x) ((void)0)
#define AMREX_IF_ON_DEVICE(x)
#define AMREX_IF_ON_HOST(x) { x }

namespace amrex {

enum class RunOn { Host, Device, Gpu = Device, Cpu = Host };
using Real = double;
using Long = long long;
constexpr Real operator""_rt(long double x) { return Real(x); }
constexpr Real operator""_rt(unsigned long long x) { return Real(x); }

[[noreturn]] inline void Abort(const std::string& m = "") {
    std::fprintf(stderr, "amrex shim abort: %s\n", m.c_str());
    std::abort();
}
[[noreturn]] inline void Error(const std::string& m = "") { Abort(m); }
inline void Warning(const std::string&) {}
template <class... T> inline void ignore_unused(const T&...) {}

// Print: an ostream that discards (the operators print diagnostics only)
struct Print {
    Print() = default;
    explicit Print(int) {}
    template <class T> Print& operator<<(const T&) { return *this; }
    Print& operator<<(std::ostream& (*)(std::ostream&)) { return *this; }
    Print& SetPrecision(int) { return *this; }
};
using AllPrint = Print;

template <class T> AMREX_FORCE_INLINE constexpr const T& max(const T& a, const T& b) { return a < b ? b : a; }
template <class T> AMREX_FORCE_INLINE constexpr const T& min(const T& a, const T& b) { return b < a ? b : a; }
template <class T, class... R> AMREX_FORCE_INLINE constexpr const T& max(const T& a, const T& b, const R&... r) { return max(max(a, b), r...); }
template <class T, class... R> AMREX_FORCE_INLINE constexpr const T& min(const T& a, const T& b, const R&... r) { return min(min(a, b), r...); }
template <class T> AMREX_FORCE_INLINE T Clamp(T v, T lo, T hi) { return v < lo ? lo : (hi < v ? hi : v); }

namespace Math {
template <class T> AMREX_FORCE_INLINE T abs(T x) { return std::abs(x); }
using std::exp; using std::log; using std::sqrt; using std::pow; using std::cos; using std::sin; using std::floor;
using std::ceil; using std::atan; using std::atan2; using std::tanh; using std::round; using std::copysign;
template <int N, class T> AMREX_FORCE_INLINE T powi(T x) { T r = T(1); for (int q = 0; q < N; ++q) r *= x; return r; }
constexpr double pi() { return 3.14159265358979323846264338327950288; }
}  // namespace Math

template <class T> using Vector = std::vector<T>;
template <class T, std::size_t N> using Array = std::array<T, N>;

struct Dim3 { int x, y, z; };

template <class T, int N>
struct GpuArray {
    T arr[N];
    AMREX_FORCE_INLINE T& operator[](int i) { return arr[i]; }
    AMREX_FORCE_INLINE const T& operator[](int i) const { return arr[i]; }
    T* data() { return arr; }
    const T* data() const { return arr; }
    static constexpr int size() { return N; }
};

template <class T, int lo, int hi>
struct Array1D {
    T arr[hi - lo + 1];
    AMREX_FORCE_INLINE T& operator()(int i) { return arr[i - lo]; }
    AMREX_FORCE_INLINE const T& operator()(int i) const { return arr[i - lo]; }
    AMREX_FORCE_INLINE T& operator[](int i) { return arr[i - lo]; }
    AMREX_FORCE_INLINE const T& operator[](int i) const { return arr[i - lo]; }
};
template <class T, int ilo, int ihi, int jlo, int jhi>
struct Array2D {
    T arr[(ihi - ilo + 1) * (jhi - jlo + 1)];
    AMREX_FORCE_INLINE T& operator()(int i, int j) { return arr[(i - ilo) + (j - jlo) * (ihi - ilo + 1)]; }
    AMREX_FORCE_INLINE const T& operator()(int i, int j) const { return arr[(i - ilo) + (j - jlo) * (ihi - ilo + 1)]; }
};

// --------------------------------------------------------------- index space
struct IntVect {
    int v[3] = {0, 0, 0};
    constexpr IntVect() = default;
    constexpr IntVect(int a, int b, int c) : v{a, b, c} {}
    explicit constexpr IntVect(int a) : v{a, a, a} {}
    AMREX_FORCE_INLINE int& operator[](int d) { return v[d]; }
    AMREX_FORCE_INLINE int operator[](int d) const { return v[d]; }
    bool operator==(const IntVect& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
    bool operator!=(const IntVect& o) const { return !(*this == o); }
    IntVect operator+(const IntVect& o) const { return {v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]}; }
    IntVect operator-(const IntVect& o) const { return {v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]}; }
    IntVect operator+(int a) const { return {v[0] + a, v[1] + a, v[2] + a}; }
    IntVect operator-(int a) const { return {v[0] - a, v[1] - a, v[2] - a}; }
    Dim3 dim3() const { return {v[0], v[1], v[2]}; }
    static IntVect TheZeroVector() { return IntVect(0); }
    static IntVect TheUnitVector() { return IntVect(1); }
    static IntVect TheDimensionVector(int d) { IntVect r; r.v[d] = 1; return r; }
    static IntVect TheNodeVector() { return IntVect(1); }
    static IntVect TheCellVector() { return IntVect(0); }
    int max() const { return std::max(v[0], std::max(v[1], v[2])); }
    int min() const { return std::min(v[0], std::min(v[1], v[2])); }
};
using GpuIntVect = IntVect;

struct IndexType {
    IntVect t;   // 1 = nodal in that direction
    IndexType() = default;
    explicit IndexType(const IntVect& a) : t(a) {}
    bool nodeCentered(int d) const { return t[d] != 0; }
    bool cellCentered(int d) const { return t[d] == 0; }
    bool cellCentered() const { return t == IntVect(0); }
    bool operator==(const IndexType& o) const { return t == o.t; }
    int operator[](int d) const { return t[d]; }
    IntVect ixType() const { return t; }
    IntVect toIntVect() const { return t; }
    static IndexType TheCellType() { return IndexType(); }
    static IndexType TheNodeType() { return IndexType(IntVect(1)); }
};

class Box {
  public:
    IntVect lo, hi;
    IndexType typ;
    Box() : lo(0), hi(-1) {}
    Box(const IntVect& l, const IntVect& h) : lo(l), hi(h) {}
    Box(const IntVect& l, const IntVect& h, const IntVect& t) : lo(l), hi(h), typ(t) {}
    Box(const IntVect& l, const IntVect& h, const IndexType& t) : lo(l), hi(h), typ(t) {}
    const IntVect& smallEnd() const { return lo; }
    const IntVect& bigEnd() const { return hi; }
    int smallEnd(int d) const { return lo[d]; }
    int bigEnd(int d) const { return hi[d]; }
    IndexType ixType() const { return typ; }
    IntVect type() const { return typ.t; }
    int type(int d) const { return typ.t[d]; }
    IntVect length() const { return {hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1}; }
    int length(int d) const { return hi[d] - lo[d] + 1; }
    Long numPts() const { return ok() ? (Long)length(0) * length(1) * length(2) : 0; }
    bool ok() const { return hi[0] >= lo[0] && hi[1] >= lo[1] && hi[2] >= lo[2]; }
    bool isEmpty() const { return !ok(); }
    bool contains(int i, int j, int k) const {
        return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
    }
    bool contains(const IntVect& p) const { return contains(p[0], p[1], p[2]); }
    bool contains(const Box& b) const { return contains(b.lo) && contains(b.hi); }
    bool intersects(const Box& b) const {
        for (int d = 0; d < 3; ++d) if (std::max(lo[d], b.lo[d]) > std::min(hi[d], b.hi[d])) return false;
        return true;
    }
    bool operator==(const Box& o) const { return lo == o.lo && hi == o.hi && typ == o.typ; }
    bool operator!=(const Box& o) const { return !(*this == o); }
    Box& setSmall(int d, int v) { lo[d] = v; return *this; }
    Box& setBig(int d, int v) { hi[d] = v; return *this; }
    Box& setSmall(const IntVect& v) { lo = v; return *this; }
    Box& setBig(const IntVect& v) { hi = v; return *this; }
    Box& setRange(int d, int l, int n = 1) { lo[d] = l; hi[d] = l + n - 1; return *this; }
    const int* loVect() const { return lo.v; }
    const int* hiVect() const { return hi.v; }
    Box& grow(int n) { for (int d = 0; d < 3; ++d) { lo[d] -= n; hi[d] += n; } return *this; }
    Box& grow(int d, int n) { lo[d] -= n; hi[d] += n; return *this; }
    Box& grow(const IntVect& n) { for (int d = 0; d < 3; ++d) { lo[d] -= n[d]; hi[d] += n[d]; } return *this; }
    Box& growLo(int d, int n = 1) { lo[d] -= n; return *this; }
    Box& growHi(int d, int n = 1) { hi[d] += n; return *this; }
    Box& shift(int d, int n) { lo[d] += n; hi[d] += n; return *this; }
    Box& shift(const IntVect& n) { lo = lo + n; hi = hi + n; return *this; }
    Box& surroundingNodes(int d) { if (typ.t[d] == 0) { typ.t[d] = 1; hi[d] += 1; } return *this; }
    Box& surroundingNodes() { for (int d = 0; d < 3; ++d) surroundingNodes(d); return *this; }
    Box& enclosedCells(int d) { if (typ.t[d] == 1) { typ.t[d] = 0; hi[d] -= 1; } return *this; }
    Box& enclosedCells() { for (int d = 0; d < 3; ++d) enclosedCells(d); return *this; }
    Box& convert(const IndexType& t) {
        for (int d = 0; d < 3; ++d) {
            if (t.t[d] == 1 && typ.t[d] == 0) hi[d] += 1;
            if (t.t[d] == 0 && typ.t[d] == 1) hi[d] -= 1;
        }
        typ = t;
        return *this;
    }
    Box& convert(const IntVect& t) { return convert(IndexType(t)); }
    Box& makeSlab(int d, int v) { lo[d] = v; hi[d] = v; return *this; }
    Box operator&(const Box& b) const {
        Box r(*this);
        for (int d = 0; d < 3; ++d) { r.lo[d] = std::max(lo[d], b.lo[d]); r.hi[d] = std::min(hi[d], b.hi[d]); }
        return r;
    }
    Box& operator&=(const Box& b) { *this = *this & b; return *this; }
    Box& refine(int) { return *this; }
    Box& coarsen(int) { return *this; }
};
AMREX_FORCE_INLINE Box surroundingNodes(Box b, int d) { return b.surroundingNodes(d); }
AMREX_FORCE_INLINE Box surroundingNodes(Box b) { return b.surroundingNodes(); }
AMREX_FORCE_INLINE Box enclosedCells(Box b) { return b.enclosedCells(); }
AMREX_FORCE_INLINE Box enclosedCells(Box b, int d) { return b.enclosedCells(d); }
AMREX_FORCE_INLINE Box convert(Box b, const IndexType& t) { return b.convert(t); }
AMREX_FORCE_INLINE Box convert(Box b, const IntVect& t) { return b.convert(t); }
AMREX_FORCE_INLINE Box grow(Box b, int n) { return b.grow(n); }
AMREX_FORCE_INLINE Box grow(Box b, int d, int n) { return b.grow(d, n); }
AMREX_FORCE_INLINE Box grow(Box b, const IntVect& n) { return b.grow(n); }
AMREX_FORCE_INLINE Box growLo(Box b, int d, int n) { return b.growLo(d, n); }
AMREX_FORCE_INLINE Box growHi(Box b, int d, int n) { return b.growHi(d, n); }
AMREX_FORCE_INLINE Box makeSlab(Box b, int d, int v) { return b.makeSlab(d, v); }
AMREX_FORCE_INLINE Box shift(Box b, int d, int n) { return b.shift(d, n); }
AMREX_FORCE_INLINE Box bdryLo(const Box& b, int d, int len = 1) {
    Box r(b); r.hi[d] = r.lo[d] + len - 1; return r;
}
AMREX_FORCE_INLINE Box bdryHi(const Box& b, int d, int len = 1) {
    Box r(b); r.lo[d] = r.hi[d] - len + 1; return r;
}
AMREX_FORCE_INLINE Dim3 lbound(const Box& b) { return b.lo.dim3(); }
AMREX_FORCE_INLINE Dim3 ubound(const Box& b) { return b.hi.dim3(); }
AMREX_FORCE_INLINE Dim3 length(const Box& b) { return b.length().dim3(); }

// --------------------------------------------------------------- Array4
template <class T>
struct Array4 {
    T* p = nullptr;
    Long jstride = 0, kstride = 0, nstride = 0;
    Dim3 begin{1, 1, 1}, end{0, 0, 0};   // end is exclusive
    int ncomp = 0;
    Array4() = default;
    Array4(T* a_p, const Dim3& b, const Dim3& e, int n) : p(a_p), begin(b), end(e), ncomp(n) {
        jstride = end.x - begin.x;
        kstride = jstride * (end.y - begin.y);
        nstride = kstride * (end.z - begin.z);
    }
    template <class U, class = typename std::enable_if<std::is_same<const U, T>::value>::type>
    Array4(const Array4<U>& o) : p(o.p), jstride(o.jstride), kstride(o.kstride), nstride(o.nstride),
                                 begin(o.begin), end(o.end), ncomp(o.ncomp) {}
    // a component slice: components [start, start+num) of another view
    template <class U, class = typename std::enable_if<std::is_same<const U, T>::value ||
                                                       std::is_same<U, T>::value>::type>
    Array4(const Array4<U>& o, int start, int num)
        : p(o.p + start * o.nstride), jstride(o.jstride), kstride(o.kstride), nstride(o.nstride), begin(o.begin),
          end(o.end), ncomp(num) {}
    AMREX_FORCE_INLINE T& operator()(int i, int j, int k) const {
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride];
    }
    AMREX_FORCE_INLINE T& operator()(int i, int j, int k, int n) const {
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
    }
    AMREX_FORCE_INLINE T& operator()(const IntVect& q, int n = 0) const { return (*this)(q[0], q[1], q[2], n); }
    T* dataPtr() const { return p; }
    T* ptr(int i, int j, int k, int n = 0) const { return &(*this)(i, j, k, n); }
    int nComp() const { return ncomp; }
    explicit operator bool() const { return p != nullptr; }
    bool contains(int i, int j, int k) const {
        return i >= begin.x && i < end.x && j >= begin.y && j < end.y && k >= begin.z && k < end.z;
    }
};
template <class T> AMREX_FORCE_INLINE Dim3 lbound(const Array4<T>& a) { return a.begin; }
template <class T> AMREX_FORCE_INLINE Dim3 ubound(const Array4<T>& a) { return {a.end.x - 1, a.end.y - 1, a.end.z - 1}; }

// --------------------------------------------------------------- loops
template <class F>
void ParallelFor(const Box& b, F&& f) {
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
        for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
}
template <class T, class F, class = typename std::enable_if<std::is_integral<T>::value>::type>
void ParallelFor(const Box& b, T ncomp, F&& f) {
    for (int n = 0; n < (int)ncomp; ++n)
        for (int k = b.lo[2]; k <= b.hi[2]; ++k)
            for (int j = b.lo[1]; j <= b.hi[1]; ++j)
                for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k, n);
}
template <class F1, class F2>
void ParallelFor(const Box& b1, const Box& b2, F1&& f1, F2&& f2) { ParallelFor(b1, f1); ParallelFor(b2, f2); }
template <class F1, class F2, class F3>
void ParallelFor(const Box& b1, const Box& b2, const Box& b3, F1&& f1, F2&& f2, F3&& f3) {
    ParallelFor(b1, f1); ParallelFor(b2, f2); ParallelFor(b3, f3);
}
template <class T, class F1, class F2, class = typename std::enable_if<std::is_integral<T>::value>::type>
void ParallelFor(const Box& b1, T n1, const Box& b2, T n2, F1&& f1, F2&& f2) {
    ParallelFor(b1, n1, f1); ParallelFor(b2, n2, f2);
}
template <class T, class F1, class F2, class F3, class = typename std::enable_if<std::is_integral<T>::value>::type>
void ParallelFor(const Box& b1, T n1, const Box& b2, T n2, const Box& b3, T n3, F1&& f1, F2&& f2, F3&& f3) {
    ParallelFor(b1, n1, f1); ParallelFor(b2, n2, f2); ParallelFor(b3, n3, f3);
}
template <class T, class F>
void ParallelFor(T n, F&& f) { for (T q = 0; q < n; ++q) f(q); }
template <class F>
void LoopOnCpu(const Box& b, F&& f) { ParallelFor(b, std::forward<F>(f)); }
template <class F>
void HostDevice_For(const Box& b, F&& f) { ParallelFor(b, std::forward<F>(f)); }
template <class F>
void For(const Box& b, F&& f) { ParallelFor(b, std::forward<F>(f)); }

namespace Gpu {
inline bool notInLaunchRegion() { return true; }
inline bool inLaunchRegion() { return false; }
inline void streamSynchronize() {}
inline void synchronize() {}
template <class T> using DeviceVector = std::vector<T>;
template <class T> using HostVector = std::vector<T>;
template <class T> using AsyncVector = std::vector<T>;
template <class T> using PinnedVector = std::vector<T>;
template <class T> using ManagedVector = std::vector<T>;
struct HostToDevice {};
struct DeviceToHost {};
struct DeviceToDevice {};
static constexpr HostToDevice hostToDevice{};
static constexpr DeviceToHost deviceToHost{};
static constexpr DeviceToDevice deviceToDevice{};
template <class Tag, class It, class Ot>
void copy(Tag, It b, It e, Ot o) { std::copy(b, e, o); }
template <class Tag, class It, class Ot>
void copyAsync(Tag, It b, It e, Ot o) { std::copy(b, e, o); }
template <class T> T* dataPtr(std::vector<T>& v) { return v.data(); }
struct KernelInfo {};
}  // namespace Gpu

inline bool TilingIfNotGPU() { return false; }

// --------------------------------------------------------------- BCRec
class BCRec {
  public:
    int bc[6] = {0, 0, 0, 0, 0, 0};
    BCRec() = default;
    BCRec(const int* l, const int* h) { for (int d = 0; d < 3; ++d) { bc[d] = l[d]; bc[d + 3] = h[d]; } }
    AMREX_FORCE_INLINE int lo(int d) const { return bc[d]; }
    AMREX_FORCE_INLINE int hi(int d) const { return bc[d + 3]; }
    const int* lo() const { return bc; }
    const int* hi() const { return bc + 3; }
    void setLo(int d, int v) { bc[d] = v; }
    void setHi(int d, int v) { bc[d + 3] = v; }
    const int* vect() const { return bc; }
};

// --------------------------------------------------------------- geometry
struct RealBox {
    Real lo_[3] = {0, 0, 0}, hi_[3] = {1, 1, 1};
    const Real* lo() const { return lo_; }
    const Real* hi() const { return hi_; }
    Real lo(int d) const { return lo_[d]; }
    Real hi(int d) const { return hi_[d]; }
};
struct RealVect {
    Real v[3] = {0, 0, 0};
    RealVect() = default;
    RealVect(Real a, Real b, Real c) : v{a, b, c} {}
    Real& operator[](int d) { return v[d]; }
    Real operator[](int d) const { return v[d]; }
};
struct Periodicity {
    IntVect period;
    static Periodicity NonPeriodic() { return {}; }
    bool isPeriodic(int d) const { return period[d] != 0; }
    bool isAnyPeriodic() const { return period[0] || period[1] || period[2]; }
};
class Arena {};
inline Arena* The_Async_Arena() { return nullptr; }
inline Arena* The_Arena() { return nullptr; }
template <class T>
class AsyncArray {
  public:
    std::vector<T> v;
    AsyncArray(const T* a, std::size_t n) : v(a, a + n) {}
    T* data() { return v.data(); }
    void copyToHost(T* h, std::size_t n) const { std::copy(v.begin(), v.begin() + n, h); }
};
struct GeometryData {
    Real prob_lo[3] = {0, 0, 0}, prob_hi[3] = {1, 1, 1}, dx[3] = {1, 1, 1};
    Box domain;
    int is_periodic[3] = {0, 0, 0};
    const Real* CellSize() const { return dx; }
    Real CellSize(int d) const { return dx[d]; }
    const Real* ProbLo() const { return prob_lo; }
    const Real* ProbHi() const { return prob_hi; }
    Real ProbLo(int d) const { return prob_lo[d]; }
    Real ProbHi(int d) const { return prob_hi[d]; }
    const Box& Domain() const { return domain; }
    int isPeriodic(int d) const { return is_periodic[d]; }
};
class Geometry {
  public:
    GeometryData g;
    Geometry() = default;
    const Box& Domain() const { return g.domain; }
    GpuArray<Real, 3> CellSizeArray() const { return {{g.dx[0], g.dx[1], g.dx[2]}}; }
    GpuArray<Real, 3> InvCellSizeArray() const { return {{1.0 / g.dx[0], 1.0 / g.dx[1], 1.0 / g.dx[2]}}; }
    GpuArray<Real, 3> ProbLoArray() const { return {{g.prob_lo[0], g.prob_lo[1], g.prob_lo[2]}}; }
    GpuArray<Real, 3> ProbHiArray() const { return {{g.prob_hi[0], g.prob_hi[1], g.prob_hi[2]}}; }
    const Real* CellSize() const { return g.dx; }
    Real CellSize(int d) const { return g.dx[d]; }
    const Real* ProbLo() const { return g.prob_lo; }
    Real ProbLo(int d) const { return g.prob_lo[d]; }
    const Real* ProbHi() const { return g.prob_hi; }
    Real ProbHi(int d) const { return g.prob_hi[d]; }
    const GeometryData& data() const { return g; }
    bool isPeriodic(int d) const { return g.is_periodic[d] != 0; }
    Periodicity periodicity() const { return {}; }
};

// --------------------------------------------------------------- containers
class BoxArray {
  public:
    std::vector<Box> boxes;
    BoxArray() = default;
    explicit BoxArray(const Box& b) : boxes{b} {}
    int size() const { return (int)boxes.size(); }
    const Box& operator[](int q) const { return boxes[q]; }
    IndexType ixType() const { return boxes.empty() ? IndexType() : boxes[0].typ; }
    BoxArray& surroundingNodes(int d) { for (auto& b : boxes) b.surroundingNodes(d); return *this; }
    BoxArray& convert(const IntVect& t) { for (auto& b : boxes) b.convert(t); return *this; }
    Box minimalBox() const { return boxes.empty() ? Box() : boxes[0]; }
};
class DistributionMapping {};
struct FabArrayBase { static inline int mfiter_tile_size[3] = {1024000, 1024000, 1024000}; };

class FArrayBox {
  public:
    Box bx;
    int nc = 0;
    std::shared_ptr<std::vector<Real>> store;   // owned or shared (aliases)
    Real* p = nullptr;
    FArrayBox() = default;
    FArrayBox(const Box& b, int n = 1, Arena* = nullptr) { resize(b, n); }
    void resize(const Box& b, int n = 1, Arena* = nullptr) {
        bx = b; nc = n;
        store = std::make_shared<std::vector<Real>>((size_t)b.numPts() * n, 0.0);
        p = store->data();
    }
    // components [scomp, scomp+n) of another FAB, sharing its storage
    void alias(const FArrayBox& o, int scomp, int n) {
        bx = o.bx; nc = n; store = o.store; p = o.p + (size_t)scomp * o.bx.numPts();
    }
    Array4<Real> array() { return Array4<Real>(p, bx.lo.dim3(), (bx.hi + 1).dim3(), nc); }
    Array4<const Real> const_array() const { return Array4<const Real>(p, bx.lo.dim3(), (bx.hi + 1).dim3(), nc); }
    Array4<const Real> array() const { return const_array(); }
    const Box& box() const { return bx; }
    int nComp() const { return nc; }
    Real* dataPtr(int n = 0) { return p + (size_t)n * bx.numPts(); }
    template <RunOn R = RunOn::Host>
    void setVal(Real v) { std::fill(p, p + (size_t)bx.numPts() * nc, v); }
    template <RunOn R = RunOn::Host>
    void setVal(Real v, const Box& b, int scomp = 0, int ncomp = 1) {
        auto a = array();
        Box r = b & bx;
        for (int n = scomp; n < scomp + ncomp; ++n) ParallelFor(r, [&](int i, int j, int k) { a(i, j, k, n) = v; });
    }
};
inline BoxArray convert(BoxArray b, const IntVect& t) { return b.convert(t); }
struct MakeType {};
static constexpr MakeType make_alias{};

}  // namespace amrex

// ---------------------------------------------------------------- enums
// AMREX_ENUM(Name, a, b, ...): an enum class; the string helpers it also
// defines in AMReX are only used by parameter parsing, which is stubbed.
#define AMREX_ENUM(CLASS, ...) enum class CLASS : int { __VA_ARGS__ }

namespace amrex {
template <class T> inline std::string getEnumNameString(const T&) { return std::string(); }
template <class T> inline std::vector<std::string> getEnumNameStrings() { return {}; }

// ParmParse: the inputs-file reader.  The operators are driven by explicit
// SolverChoice fields here, so every query reports "not found".
class ParmParse {
  public:
    ParmParse() = default;
    explicit ParmParse(const std::string&) {}
    template <class T> int query(const char*, T&, int = 0) const { return 0; }
    template <class T> int query(const std::string&, T&, int = 0) const { return 0; }
    template <class T> void get(const char*, T&, int = 0) const {}
    template <class T> int queryarr(const char*, T&, int = 0, int = 0) const { return 0; }
    template <class T> int queryarr(const std::string&, T&, int = 0, int = 0) const { return 0; }
    template <class T> void getarr(const char*, T&, int = 0, int = 0) const {}
    template <class T> int query_enum_case_insensitive(const char*, T&, int = 0) const { return 0; }
    template <class T> int query_enum_case_insensitive(const std::string&, T&, int = 0) const { return 0; }
    template <class T> int query_enum_sloppy(const char*, T&, const std::string& = "", int = 0) const { return 0; }
    template <class T> void get_enum_case_insensitive(const char*, T&, int = 0) const {}
    template <class T> int queryAdd(const char*, T&) const { return 0; }
    template <class T> void add(const char*, const T&) const {}
    template <class T> void addarr(const char*, const T&) const {}
    template <class T> int queryWithParser(const char*, T&) const { return 0; }
    int countval(const char*, int = 0) const { return 0; }
    std::string prefixedName(const std::string& s) const { return s; }
    std::string getPrefix() const { return std::string(); }
    bool contains(const char*) const { return false; }
};
}  // namespace amrex

// --------------------------------------------------------------- MultiFab
// One FAB covering the box of a one-box BoxArray plus its ghost cells.  The
// domain's lateral periodicity for FillBoundary is set by the harness.
namespace amrex {
struct ShimDomain {
    static inline Box domain;                 // cell-centred problem domain
    static inline int periodic[3] = {1, 1, 0};
};
class MultiFab;
class MFIter {
  public:
    const MultiFab* m;
    bool ok = true;
    explicit MFIter(const MultiFab& a, bool = false) : m(&a) {}
    MFIter(const MultiFab& a, const IntVect&) : m(&a) {}
    bool isValid() const { return ok; }
    MFIter& operator++() { ok = false; return *this; }
    int index() const { return 0; }
    int LocalIndex() const { return 0; }
    Box validbox() const;
    Box tilebox() const { return validbox(); }
    Box tilebox(const IntVect& nodal) const {
        Box b = validbox();
        Box c = b; c.enclosedCells();
        c.convert(nodal);
        return c;
    }
    Box tilebox(const IntVect& nodal, const IntVect& ng) const { return grow(tilebox(nodal), ng); }
    Box nodaltilebox(int d) const { Box b = validbox(); b.enclosedCells(); return b.surroundingNodes(d); }
    Box growntilebox(int ng = -1000) const;
    Box growntilebox(const IntVect& ng) const { return grow(validbox(), ng); }
    Box grownnodaltilebox(int d, int ng) const { return grow(nodaltilebox(d), ng); }
    Box fabbox() const;
};
class MultiFab {
  public:
    BoxArray ba;
    int nc = 0;
    IntVect ng;
    FArrayBox fab;
    MultiFab() = default;
    MultiFab(const BoxArray& b, const DistributionMapping&, int n, int g) { define(b, n, IntVect(g)); }
    MultiFab(const BoxArray& b, const DistributionMapping&, int n, const IntVect& g) { define(b, n, g); }
    MultiFab(const MultiFab& o, MakeType, int scomp, int n) : ba(o.ba), nc(n), ng(o.ng) { fab.alias(o.fab, scomp, n); }
    void define(const BoxArray& b, const DistributionMapping&, int n, int g) { define(b, n, IntVect(g)); }
    void define(const BoxArray& b, int n, const IntVect& g) {
        ba = b; nc = n; ng = g;
        Box fb = ba[0];
        fb.grow(g);
        fab.resize(fb, n);
    }
    int nComp() const { return nc; }
    int nGrow() const { return ng[0]; }
    IntVect nGrowVect() const { return ng; }
    const BoxArray& boxArray() const { return ba; }
    DistributionMapping DistributionMap() const { return {}; }
    IndexType ixType() const { return ba.ixType(); }
    Array4<Real> array(const MFIter&) { return fab.array(); }
    Array4<const Real> array(const MFIter&) const { return fab.const_array(); }
    Array4<const Real> const_array(const MFIter&) const { return fab.const_array(); }
    Array4<Real> array(int) { return fab.array(); }
    Array4<const Real> const_array(int) const { return fab.const_array(); }
    FArrayBox& operator[](const MFIter&) { return fab; }
    const FArrayBox& operator[](const MFIter&) const { return fab; }
    FArrayBox& get(const MFIter&) { return fab; }
    void setVal(Real v) { fab.setVal(v); }
    void setVal(Real v, int scomp, int n, int g = 0) { setVal(v, scomp, n, IntVect(g)); }
    void setVal(Real v, int scomp, int n, const IntVect& g) {
        Box b = ba[0]; b.grow(g);
        fab.setVal(v, b, scomp, n);
    }
    // periodic images into the ghost cells (x and y periodic, one box)
    void FillBoundary(const Periodicity& = Periodicity()) { FillBoundary(0, nc); }
    void FillBoundary(int scomp, int n, const Periodicity& = Periodicity()) {
        const Box& dom = ShimDomain::domain;
        Box v = ba[0];
        Box g = fab.bx;
        auto a = fab.array();
        int len[3];
        for (int d = 0; d < 3; ++d) len[d] = dom.length(d);
        ParallelFor(g, [&](int i, int j, int k) {
            if (v.contains(i, j, k)) return;
            int s[3] = {i, j, k};
            for (int d = 0; d < 2; ++d) {
                if (!ShimDomain::periodic[d]) continue;
                while (s[d] < v.lo[d]) s[d] += len[d];
                while (s[d] > v.hi[d]) s[d] -= len[d];
            }
            if (!v.contains(s[0], s[1], s[2])) return;
            for (int q = scomp; q < scomp + n; ++q) a(i, j, k, q) = a(s[0], s[1], s[2], q);
        });
    }
    static void Copy(MultiFab& dst, const MultiFab& src, int sc, int dc, int n, int g) {
        Copy(dst, src, sc, dc, n, IntVect(g));
    }
    static void Copy(MultiFab& dst, const MultiFab& src, int sc, int dc, int n, const IntVect& g) {
        Box b = dst.ba[0]; b.grow(g);
        auto d = dst.fab.array();
        auto s = src.fab.const_array();
        for (int q = 0; q < n; ++q) ParallelFor(b, [&](int i, int j, int k) { d(i, j, k, dc + q) = s(i, j, k, sc + q); });
    }
};
inline Box MFIter::validbox() const { return m->ba[0]; }
inline Box MFIter::growntilebox(int g) const { return grow(m->ba[0], g == -1000 ? m->ng : IntVect(g)); }
inline Box MFIter::fabbox() const { return m->fab.bx; }
using iMultiFab = MultiFab;
inline std::unique_ptr<iMultiFab> OwnerMask(const MultiFab&, const Periodicity&, const IntVect& = IntVect(0)) {
    return nullptr;
}
class YAFluxRegister {};
}  // namespace amrex
