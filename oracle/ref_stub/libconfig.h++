// Minimal stand-in for <libconfig.h++>: the harness fills the reference's
// namespace globals directly, so only the type names have to exist.
#ifndef ASD_REF_STUB_LIBCONFIG_HPP
#define ASD_REF_STUB_LIBCONFIG_HPP
namespace libconfig {
class Setting {};
class Config {};
class SettingNotFoundException { public: const char* getPath() const { return ""; } };
}
#endif
