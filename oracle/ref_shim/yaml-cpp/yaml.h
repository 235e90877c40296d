/* Minimal stand-in for yaml-cpp: the reference headers only name YAML::Node
 * in read_config methods that the oracle pins never call. */
#ifndef ORACLE_SHIM_YAML_H
#define ORACLE_SHIM_YAML_H
namespace YAML {
struct Node {
    Node operator[](int) const { return Node(); }
    Node operator[](const char *) const { return Node(); }
    template <typename T> T as() const { return T(); }
};
}  // namespace YAML
#endif
