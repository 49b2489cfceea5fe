// payloads_ref.cpp -- writes component payloads with the reference's own POD types (test fixture generator).
//
// Built by tests/golden/make_payloads.py against a Piper2 checkout (-I <Piper2>/Src); never part of the
// library.  Reads one request per line on stdin, fills the reference's payload struct named by the request
// from the numbers that follow, and prints "<sizeof> <hex bytes>".  Handles (TraversalHandle, CallHandle,
// StatisticsHandle) are given as integers and stored as the pointer values the reference keeps.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "BuiltinComponent/Geometry/BasicShapes/Shared.hpp"
#include "BuiltinComponent/Integrator/PathTracing/Shared.hpp"
#include "BuiltinComponent/Light/AreaLight/Shared.hpp"
#include "BuiltinComponent/Light/BasicLight/Shared.hpp"
#include "BuiltinComponent/RenderDriver/FixedSampler/Shared.hpp"
#include "BuiltinComponent/Sensor/PerspectiveCamera/Shared.hpp"
#include "BuiltinComponent/Surface/Classic/Shared.hpp"
#include "BuiltinComponent/Texture/ProceduralTexture/Shared.hpp"

using namespace Piper;

namespace {

template <class T>
void emit(const T& v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    std::printf("%zu ", sizeof(T));
    for (size_t i = 0; i < sizeof(T); ++i) std::printf("%02x", p[i]);
    std::printf("\n");
}

template <class H>
H handle(std::istream& in) {
    unsigned long long v;
    in >> v;
    return reinterpret_cast<H>(static_cast<uintptr_t>(v));
}

float num(std::istream& in) {
    double v;
    in >> v;
    return static_cast<float>(v);
}

template <class F>
Call<F> call(std::istream& in) {
    return Call<F>{ handle<CallHandle>(in) };
}

}  // namespace

int main() {
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        std::string kind;
        in >> kind;
        if (kind == "constant") {  // ConstantData: channel, value[4]
            ConstantData d{};
            in >> d.channel;
            for (auto& v : d.value) v = Dimensionless<float>{ num(in) };
            emit(d);
        } else if (kind == "matte") {
            MatteData d{ call<TextureSampleFunc>(in), call<TextureSampleFunc>(in) };
            emit(d);
        } else if (kind == "plastic") {
            PlasticData d{ call<TextureSampleFunc>(in), call<TextureSampleFunc>(in), call<TextureSampleFunc>(in) };
            emit(d);
        } else if (kind == "glass") {
            GlassData d{ call<TextureSampleFunc>(in), call<TextureSampleFunc>(in), call<TextureSampleFunc>(in),
                         call<TextureSampleFunc>(in) };
            emit(d);
        } else if (kind == "mirror") {
            MirrorData d{ call<TextureSampleFunc>(in) };
            emit(d);
        } else if (kind == "substrate") {
            SubstrateData d{ call<TextureSampleFunc>(in), call<TextureSampleFunc>(in), call<TextureSampleFunc>(in),
                             call<TextureSampleFunc>(in) };
            emit(d);
        } else if (kind == "environment") {  // SampledEnvironmentData: traversal, radiance rgb
            SampledEnvironmentData d{};
            d.traversal = handle<TraversalHandle>(in);
            d.texture.r = Radiance{ num(in) };
            d.texture.g = Radiance{ num(in) };
            d.texture.b = Radiance{ num(in) };
            emit(d);
        } else if (kind == "plane") {  // PerPlaneData: origin, u, v, normal, tangent, maxDetComp
            PerPlaneData d{};
            d.origin = { Distance{ num(in) }, Distance{ num(in) }, Distance{ num(in) } };
            d.u = { Distance{ num(in) }, Distance{ num(in) }, Distance{ num(in) } };
            d.v = { Distance{ num(in) }, Distance{ num(in) }, Distance{ num(in) } };
            const float n0 = num(in), n1 = num(in), n2 = num(in);
            d.normal = Normal<float, FOR::Local>{ Vector<Dimensionless<float>, FOR::Local>{ { n0 }, { n1 }, { n2 } },
                                                  Unsafe{} };
            const float t0 = num(in), t1 = num(in), t2 = num(in);
            d.tangent = Normal<float, FOR::Local>{ Vector<Dimensionless<float>, FOR::Local>{ { t0 }, { t1 }, { t2 } },
                                                   Unsafe{} };
            in >> d.maxDetComp;
            emit(d);
        } else if (kind == "cdf") {  // CDFData: primitives, traversal, cdf, pdf, inverseArea, size
            CDFData d{};
            in >> d.primitives;
            d.traversal = handle<TraversalHandle>(in);
            in >> d.cdf >> d.pdf;
            d.inverseArea = Dimensionless<float>{ num(in) };
            in >> d.size;
            emit(d);
        } else if (kind == "diffuse") {  // DiffuseAreaLightData: radiance rgb, sample call, area
            DiffuseAreaLightData d{};
            d.radiance.r = Radiance{ num(in) };
            d.radiance.g = Radiance{ num(in) };
            d.radiance.b = Radiance{ num(in) };
            d.sample = call<GeometrySampleFunc>(in);
            d.area = Area<float>{ num(in) };
            emit(d);
        } else if (kind == "camera") {  // PCData: traversal, lookAt, size (m), upRef, focalLength, apertureRadius
            PCData d{};
            d.traversal = handle<TraversalHandle>(in);
            d.lookAt = { Distance{ num(in) }, Distance{ num(in) }, Distance{ num(in) } };
            d.size.x = num(in);
            d.size.y = num(in);
            const float u0 = num(in), u1 = num(in), u2 = num(in);
            d.upRef = Normal<float, FOR::World>{ Vector<Dimensionless<float>, FOR::World>{ { u0 }, { u1 }, { u2 } },
                                                 Unsafe{} };
            d.focalLength = Distance{ num(in) };
            d.apertureRadius = Distance{ num(in) };
            emit(d);
        } else if (kind == "pathtracing") {  // Data: maxDepth, minDepthForRussianRoulette, 3 statistics handles
            Data d{};
            in >> d.maxDepth >> d.minDepthForRussianRoulette;
            d.profileDepth = handle<StatisticsHandle>(in);
            d.profilePathTime = handle<StatisticsHandle>(in);
            d.profileValidRay = handle<StatisticsHandle>(in);
            emit(d);
        } else if (kind == "driver") {  // RDData: filter call
            RDData d{ call<FilterFunc>(in) };
            emit(d);
        } else if (kind == "gaussian") {  // GaussianFilterData: negAlpha, sub
            GaussianFilterData d{ num(in), num(in) };
            emit(d);
        } else if (!kind.empty()) {
            std::fprintf(stderr, "unknown request %s\n", kind.c_str());
            return 1;
        }
    }
    return 0;
}
