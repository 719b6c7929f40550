/* Stand-in for OpenColorIO used only to compile the reference's golden
 * generator.  The display-encode fixture it feeds is outside the raw->linear
 * path, so the processor is an identity.  Test infrastructure only. */
#pragma once
#include <memory>
#define OCIO_NAMESPACE OCIO_STUB
namespace OCIO_STUB {
struct PackedImageDesc {
    PackedImageDesc(float*, long, long, long) {}
};
struct CPUProcessor {
    void apply(PackedImageDesc&) const {}
};
struct Processor {
    std::shared_ptr<const CPUProcessor> getDefaultCPUProcessor() const {
        return std::make_shared<CPUProcessor>();
    }
};
struct Config {
    static std::shared_ptr<const Config> CreateFromFile(const char*) {
        return std::make_shared<Config>();
    }
    std::shared_ptr<const Processor> getProcessor(const char*, const char*) const {
        return std::make_shared<Processor>();
    }
};
}  // namespace OCIO_STUB
