#pragma once
// JSON-with-comments configuration (API of the reference's
// include/IO/ConfigFile.h; needs nlohmann/json on the include path).
#include <string>

#include <nlohmann/json.hpp>

namespace PhiX {
namespace IO {
class ConfigFile {
public:
    explicit ConfigFile(const std::string& path);
    static ConfigFile fromArgs(int argc, char* argv[], const std::string& defaultPath = "settings/settings.jsonc");
    const nlohmann::json& operator[](const std::string& key) const;
    bool has(const std::string& key) const;
    const nlohmann::json& data() const { return data_; }

private:
    nlohmann::json data_;
    static std::string stripLineComment(const std::string& line);
};
}  // namespace IO
}  // namespace PhiX
