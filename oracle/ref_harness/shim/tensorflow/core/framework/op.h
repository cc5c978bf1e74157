// Minimal stand-ins for the TensorFlow op-registration API, just enough for
// the op-wrapper half of the reference's temporal.cu.cc to compile next to
// its kernel (test infrastructure; nothing here is called).
#pragma once
#include <cstdint>
#include <initializer_list>
#include <cuda_runtime.h>
#include "unsupported/Eigen/CXX11/Tensor"
namespace tensorflow {
struct Status {};
struct TensorShape {
    int64_t d[8] = {0};
    int n = 0;
    TensorShape() = default;
    TensorShape(std::initializer_list<int64_t> l) { for (auto v : l) d[n++] = v; }
    int64_t dim_size(int i) const { return d[i]; }
};
template <typename T> struct FlatStub {
    T *p;
    T *data() const { return p; }
};
struct Tensor {
    TensorShape s;
    void *p = nullptr;
    const TensorShape &shape() const { return s; }
    template <typename T> FlatStub<T> flat() const { return FlatStub<T>{static_cast<T *>(p)}; }
};
class OpKernelConstruction {
  public:
    template <typename T> Status GetAttr(const char *, T *) { return Status(); }
};
class OpKernelContext {
  public:
    Tensor input(int) { return Tensor(); }
    template <typename D> const D &eigen_device() { static const D d(nullptr); return d; }
    Status allocate_output(int, const TensorShape &, Tensor **) { return Status(); }
};
class OpKernel {
  public:
    explicit OpKernel(OpKernelConstruction *) {}
    virtual ~OpKernel() {}
    virtual void Compute(OpKernelContext *) = 0;
};
namespace shape_inference {
struct ShapeHandle {};
struct DimensionHandle {
    DimensionHandle() = default;
    DimensionHandle(int64_t) {}
};
struct InferenceContext {
    ShapeHandle input(int) { return ShapeHandle(); }
    DimensionHandle Dim(ShapeHandle, int) { return DimensionHandle(); }
    void set_output(int, ShapeHandle) {}
    ShapeHandle MakeShape(std::initializer_list<DimensionHandle>) { return ShapeHandle(); }
};
}  // namespace shape_inference
struct OpDefBuilderStub {
    explicit OpDefBuilderStub(const char *) {}
    OpDefBuilderStub &Input(const char *) { return *this; }
    OpDefBuilderStub &Output(const char *) { return *this; }
    OpDefBuilderStub &Attr(const char *) { return *this; }
    template <typename F> OpDefBuilderStub &SetShapeFn(F) { return *this; }
};
}  // namespace tensorflow
#define CD_STUB_CAT2(a, b) a##b
#define CD_STUB_CAT(a, b) CD_STUB_CAT2(a, b)
#define REGISTER_OP(name) \
    static ::tensorflow::OpDefBuilderStub CD_STUB_CAT(cd_stub_op_, __COUNTER__) = ::tensorflow::OpDefBuilderStub(name)
#define REGISTER_KERNEL_BUILDER(...)
#define OP_REQUIRES_OK(ctx, expr) \
    do { (void)(expr); } while (0)
