// pybind11 module spyker_b200_plugin: the reference's compiled plugin
// (src/bind/bind.cpp:110-407, module spyker_plugin) for the dense hot path,
// bound to the C++ Spyker:: layer of spyker_b200.hpp.  Same names and
// argument order as the plugin: tensors come in as device tensors (made from
// NumPy arrays, or views of a device pointer such as torch's data_ptr()),
// ops write into the caller's output tensors where the plugin does, and
// shapes travel as lists of 1, 2 or 4 values (the plugin's Expand2/Expand4).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstring>
#include <map>
#include <string>

#include "spyker_b200.hpp"

namespace py = pybind11;
using namespace Spyker;

namespace
{
// The plugin's type names (bind.cpp str2type).
Type str2type(const std::string &s)
{
    static const std::map<std::string, Type> m = {{"i8", Type::I8},   {"i16", Type::I16}, {"i32", Type::I32},
                                                  {"i64", Type::I64}, {"u8", Type::U8},   {"u16", Type::U16},
                                                  {"u32", Type::U32}, {"u64", Type::U64}, {"f16", Type::F16},
                                                  {"f32", Type::F32}, {"f64", Type::F64}};
    auto it = m.find(s);
    if (it == m.end()) throw Error("Unknown data type " + s + ".");
    return it->second;
}

std::string type2str(Type t)
{
    static const char *names[] = {"i8", "i16", "i32", "i64", "u8", "u16", "u32", "u64", "f16", "f32", "f64"};
    return names[int(t)];
}

Expand2 e2(const Shape &s)
{
    if (s.size() == 1) return Expand2(s[0]);
    if (s.size() == 2) return Expand2(s[0], s[1]);
    throw Error("Expected 1 or 2 values.");
}

Expand4 e4(const Shape &s)
{
    if (s.size() == 1) return Expand4(s[0]);
    if (s.size() == 2) return Expand4(s[0], s[1]);
    if (s.size() == 4) return Expand4(s[0], s[1], s[2], s[3]);
    throw Error("Expected 1, 2 or 4 values.");
}

py::dtype np_dtype(Type t)
{
    switch (t)
    {
    case Type::I8: return py::dtype::of<int8_t>();
    case Type::I16: return py::dtype::of<int16_t>();
    case Type::I32: return py::dtype::of<int32_t>();
    case Type::I64: return py::dtype::of<int64_t>();
    case Type::U8: return py::dtype::of<uint8_t>();
    case Type::U16: return py::dtype::of<uint16_t>();
    case Type::U32: return py::dtype::of<uint32_t>();
    case Type::U64: return py::dtype::of<uint64_t>();
    case Type::F32: return py::dtype::of<float>();
    case Type::F64: return py::dtype::of<double>();
    default: throw Error("Unsupported NumPy type.");
    }
}

Type np_type(const py::array &a)
{
    const py::dtype d = a.dtype();
    if (d.is(py::dtype::of<uint8_t>())) return Type::U8;
    if (d.is(py::dtype::of<float>())) return Type::F32;
    if (d.is(py::dtype::of<double>())) return Type::F64;
    if (d.is(py::dtype::of<int32_t>())) return Type::I32;
    if (d.is(py::dtype::of<int64_t>())) return Type::I64;
    if (d.is(py::dtype::of<uint16_t>())) return Type::U16;
    if (d.is(py::dtype::of<int16_t>())) return Type::I16;
    if (d.is(py::dtype::of<int8_t>())) return Type::I8;
    throw Error("Unsupported NumPy type.");
}

Tensor from_numpy(py::array a)
{
    a = py::array::ensure(a, py::array::c_style);
    Shape shape(a.shape(), a.shape() + a.ndim());
    return Tensor::from_host(a.data(), np_type(a), shape);
}

py::array to_numpy(const Tensor &t)
{
    py::array a(np_dtype(t.type()), t.shape());
    if (t.numel() > 0) t.to_host(a.mutable_data());
    return a;
}
}  // namespace

PYBIND11_MODULE(spyker_b200_plugin, m)
{
    m.doc() = "spyker_b200 plugin: the reference's spyker_plugin surface for the dense hot path on the GPU";
    py::register_exception<Error>(m, "SpykerError");

    py::class_<Tensor>(m, "Tensor")
        .def_property_readonly("shape", [](const Tensor &t) { return t.shape(); })
        .def_property_readonly("type", [](const Tensor &t) { return type2str(t.type()); })
        .def_property_readonly("data", [](const Tensor &t) { return reinterpret_cast<uintptr_t>(t.data()); })
        .def("numel", &Tensor::numel)
        .def("numpy", &to_numpy);
    // bind.cpp:181-188: a new device tensor, or a view of device memory
    m.def("tensor", [](std::string type, Shape shape) { return Tensor(str2type(type), shape); });
    m.def("tensor", [](uintptr_t data, std::string type, Shape shape) {
        return Tensor(reinterpret_cast<void *>(data), str2type(type), shape);
    });
    m.def("from_numpy", &from_numpy);

    py::class_<Winner>(m, "Winner")
        .def_readonly("c", &Winner::c)
        .def_readonly("t", &Winner::t)
        .def_readonly("z", &Winner::z)
        .def_readonly("y", &Winner::y)
        .def_readonly("x", &Winner::x);
    py::class_<DoGFilter>(m, "DoGFilter")
        .def(py::init<F64, F64>())
        .def_readwrite("std1", &DoGFilter::std1)
        .def_readwrite("std2", &DoGFilter::std2);
    py::class_<STDPConfig>(m, "STDPConfig")
        .def(py::init<F64, F64, bool, F64, F64>(), py::arg("positive"), py::arg("negative"),
             py::arg("stabilize") = true, py::arg("lower") = 0.0, py::arg("upper") = 1.0)
        .def_readwrite("positive", &STDPConfig::positive)
        .def_readwrite("negative", &STDPConfig::negative)
        .def_readwrite("stabilize", &STDPConfig::stabilize)
        .def_readwrite("lower", &STDPConfig::lower)
        .def_readwrite("upper", &STDPConfig::upper);

    py::class_<GaborFilter>(m, "GaborFilter")
        .def(py::init<F64, F64, F64, F64, F64>())
        .def_readwrite("sigma", &GaborFilter::sigma)
        .def_readwrite("theta", &GaborFilter::theta)
        .def_readwrite("gamma", &GaborFilter::gamma)
        .def_readwrite("lambda_", &GaborFilter::lambda)
        .def_readwrite("psi", &GaborFilter::psi);
    py::class_<BPConfig>(m, "BPConfig")
        .def(py::init<>())
        .def(py::init<float, float, float, float>())
        .def_readwrite("sfactor", &BPConfig::sfactor)
        .def_readwrite("lrate", &BPConfig::lrate)
        .def_readwrite("lrf", &BPConfig::lrf)
        .def_readwrite("lamda", &BPConfig::lambda);

    // bind.cpp:241-250: event lists on the device
    py::class_<SparseTensor>(m, "SparseTensor")
        .def(py::init<Tensor, F64>(), py::arg("tensor"), py::arg("threshold") = 0.0)
        .def_property_readonly("numel", &SparseTensor::numel)
        .def_property_readonly("dims", [](const SparseTensor &t) { return Size(t.shape.size()); })
        .def_property_readonly("shape", [](const SparseTensor &t) { return t.shape; })
        .def_property_readonly("capacity", &SparseTensor::capacity)
        .def("__bool__", [](const SparseTensor &t) { return t.offsets.valid(); })
        .def("dense", &SparseTensor::dense)
        .def("sparsity", &SparseTensor::sparsity);

    py::class_<DoG>(m, "DoG")
        .def(py::init([](Size size, const std::vector<DoGFilter> &filters, Shape pad) {
            return DoG(size, filters, e4(pad));
        }))
        .def_readwrite("kernel", &DoG::kernel)
        .def("_forward", [](DoG &layer, Tensor input) { return layer(input); });

    py::class_<Gabor>(m, "Gabor")
        .def(py::init([](Size size, const std::vector<GaborFilter> &filters, Shape pad) {
            return Gabor(size, filters, e4(pad));
        }))
        .def_readwrite("kernel", &Gabor::kernel)
        .def("_forward", [](Gabor &layer, Tensor input) { return layer(input); });
    py::class_<LoG>(m, "LoG")
        .def(py::init([](Size size, const std::vector<F64> &stds, Shape pad) { return LoG(size, stds, e4(pad)); }))
        .def_readwrite("kernel", &LoG::kernel)
        .def("_forward", [](LoG &layer, Tensor input) { return layer(input); });

    py::class_<FC>(m, "FC")
        .def(py::init([](Size input, Size output, F64 mean, F64 std) { return FC(input, output, mean, std); }))
        .def_readwrite("kernel", &FC::kernel)
        .def_readwrite("stdpconfig", &FC::stdpconfig)
        .def_readwrite("bpconfig", &FC::bpconfig)
        .def("_forward", [](FC &layer, Tensor input, Tensor output, bool sign) { return layer(input, output, sign); })
        .def("_stdp", [](FC &layer, Tensor input, const Winners &winners, Tensor output) {
            layer.stdp(input, winners, output);
        })
        .def("_backward", [](FC &layer, Tensor input, Tensor output, Tensor grad, Tensor next) {
            layer.backward(input, output, grad, next);
        });

    py::class_<Conv>(m, "Conv")
        .def(py::init([](Size input, Size output, Shape kernel, Shape stride, Shape pad, F64 mean, F64 std) {
            return Conv(input, output, e2(kernel), e2(stride), e4(pad), mean, std);
        }))
        .def_readwrite("kernel", &Conv::kernel)
        .def_readwrite("stdpconfig", &Conv::stdpconfig)
        .def_readwrite("precision", &Conv::precision)
        .def("_forward", [](Conv &layer, Tensor input, Tensor output) {
            conv(input, layer.kernel, output, layer.stride(), layer.pad(), layer.precision);
        })
        .def("_forward", [](Conv &layer, SparseTensor input, F64 threshold) { return layer(input, threshold); })
        .def("_stdp", [](Conv &layer, Tensor input, const Winners &winners, Tensor output) {
            layer.stdp(input, winners, output);
        })
        .def("_stdp", [](Conv &layer, SparseTensor input, const Winners &winners) { layer.stdp(input, winners); });

    // bind.cpp:365-392, the dense hot path
    m.def("conv", [](Tensor input, Tensor kernel, Tensor output, Shape stride, Shape pad) {
        conv(input, kernel, output, e2(stride), e4(pad));
    });
    m.def("pad", [](Tensor input, Tensor output, Shape pad4, F64 value) {
        Tensor out = pad(input, e4(pad4), value);
        detail::require(out.shape() == output.shape() && out.type() == output.type(), "Output shape or type differs.");
        detail::cuda(cudaMemcpyAsync(output.data(), out.data(), out.bytes(), cudaMemcpyDeviceToDevice, stream()),
                     "pad");
    });
    m.def("threshold", [](Tensor input, F64 threshold, F64 value) { Spyker::threshold(input, threshold, value, true); });
    m.def("code", [](Tensor input, Tensor output, Size time, bool sort, std::string code) {
        if (code != "rank") throw Error("The plugin's dense path takes the rank code.");
        Spyker::code(input, output, time, sort);
    });
    m.def("infinite", [](Tensor input, F64 value) { Spyker::infinite(input, value, true); });
    m.def("fire", [](Tensor input, Tensor output, F64 threshold, std::string code) {
        if (code != "rank") throw Error("The plugin's dense path takes the rank code.");
        Spyker::fire(input, output, threshold);
    });
    m.def("gather", [](Tensor input, Tensor output, F64 threshold, std::string code) {
        if (code != "rank") throw Error("The plugin's dense path takes the rank code.");
        Spyker::gather(input, output, threshold);
    });
    m.def("pool", [](Tensor input, Tensor output, Shape kernel, Shape stride, Shape pad) {
        Spyker::pool(input, output, e2(kernel), stride.empty() ? Expand2(0) : e2(stride),
                     pad.empty() ? Expand4(0) : e4(pad));
    });
    m.def("inhibit", [](Tensor input, F64 threshold) { Spyker::inhibit(input, threshold, true); });
    m.def("fcwta", [](Tensor input, Size radius, Size count, F64 threshold) {
        return Spyker::fcwta(input, radius, count, threshold);
    });
    m.def("convwta", [](Tensor input, Shape radius, Size count, F64 threshold) {
        return Spyker::convwta(input, e2(radius), count, threshold);
    });
    m.def("fc", [](Tensor input, Tensor kernel, Tensor output, bool sign) { Spyker::fc(input, kernel, output, sign); });
    m.def("scatter", [](Tensor input, Tensor output) {
        detail::require(output.dims() >= 2, "Output dimensions must be at least 2.");
        Tensor out = Spyker::scatter(input, output.shape(1), output.type());
        detail::require(out.shape() == output.shape(), "Output shape is not compatible with the input.");
        detail::cuda(cudaMemcpyAsync(output.data(), out.data(), out.bytes(), cudaMemcpyDeviceToDevice, stream()),
                     "scatter");
    });
    m.def("backward", [](Tensor input, Tensor output, Tensor target, Size time, F64 gamma) {
        Spyker::backward(input, output, target, time, gamma);
    });
    m.def("labelize", [](Tensor input, Tensor output, F64 threshold) { Spyker::labelize(input, output, threshold); });

    // bind.cpp:396-407, the event-list path
    py::module_ sp = m.def_submodule("sparse");
    sp.def("conv", [](SparseTensor input, Tensor kernel, F64 threshold, Shape stride, Shape pad) {
        return Sparse::conv(input, kernel, threshold, e2(stride), e4(pad));
    });
    sp.def("pad", [](SparseTensor input, Shape pad) { return Sparse::pad(input, e4(pad)); });
    sp.def("code", [](Tensor input, Size time, bool sort) { return Sparse::code(input, time, sort); });
    sp.def("gather", [](SparseTensor input, std::string type) { return Sparse::gather(input, str2type(type)); });
    sp.def("pool", [](SparseTensor input, Shape kernel, Shape stride, Shape pad) {
        return Sparse::pool(input, e2(kernel), stride.empty() ? Expand2(0) : e2(stride),
                            pad.empty() ? Expand4(0) : e4(pad));
    });
    sp.def("inhibit", [](SparseTensor input) { return Sparse::inhibit(input); });
    sp.def("convwta", [](SparseTensor input, Shape radius, Size count) {
        return Sparse::convwta(input, e2(radius), count);
    });

    // no counterpart in the plugin: the fused layer
    m.def("conv_fire_wta", [](Tensor input, Conv &layer, F64 threshold, Shape radius, Size count, Shape pool) {
        LayerOutput r = Spyker::conv_fire_wta(input, layer, threshold, e2(radius), count,
                                              pool.empty() ? Expand2(0) : e2(pool));
        return py::make_tuple(r.spikes, r.winners, r.pooled.valid() ? py::cast(r.pooled) : py::none());
    });
    m.def("synchronize", &Spyker::synchronize);
    m.attr("CONV_FP32") = int(SPK_CONV_FP32);
    m.attr("CONV_BF16X2") = int(SPK_CONV_BF16X2);
    m.attr("CONV_BF16X3") = int(SPK_CONV_BF16X3);
}
