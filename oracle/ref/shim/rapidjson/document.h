// Stand-in for rapidjson (absent here): the reference's headers name these
// types in declarations of its JSON import / export, which the harness in
// oracle/ref never calls.
#pragma once
namespace rapidjson {
class Document;
class Value;
class StringBuffer;
template <class OutputStream, class... Rest>
class Writer;
}  // namespace rapidjson
