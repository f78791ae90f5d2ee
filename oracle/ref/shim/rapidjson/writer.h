// Stand-in for rapidjson (absent here), so that the reference's sources
// compile: the members its JSON import / export names (cipher_t.cpp:42-81,
// ckkscontext.cpp:50-100), each of which aborts if called.  The harness in
// oracle/ref never calls that import / export.  Test infrastructure only.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>

namespace rapidjson {

[[noreturn]] inline void json_stand_in_called(const char* what) {
  std::fprintf(stderr, "rapidjson stand-in: %s is not available in this harness\n", what);
  std::abort();
}

struct Allocator {};

class Value {
 public:
  Value() {}
  Value& SetObject() { json_stand_in_called("Value::SetObject"); }
  Value& SetArray() { json_stand_in_called("Value::SetArray"); }
  template <class... A>
  Value& SetString(A&&...) { json_stand_in_called("Value::SetString"); }
  template <class N, class V>
  Value& AddMember(N&&, V&&, Allocator&) { json_stand_in_called("Value::AddMember"); }
  template <class V>
  Value& PushBack(V&&, Allocator&) { json_stand_in_called("Value::PushBack"); }
  Value& operator[](const char*) { json_stand_in_called("Value::operator[]"); }
  const Value& operator[](const char*) const { json_stand_in_called("Value::operator[]"); }
  const char* GetString() const { json_stand_in_called("Value::GetString"); }
  int GetInt() const { json_stand_in_called("Value::GetInt"); }
  int64_t GetInt64() const { json_stand_in_called("Value::GetInt64"); }
  uint64_t GetUint64() const { json_stand_in_called("Value::GetUint64"); }
  double GetDouble() const { json_stand_in_called("Value::GetDouble"); }
  bool HasMember(const char*) const { json_stand_in_called("Value::HasMember"); }
};

class Document : public Value {
 public:
  Allocator& GetAllocator() { json_stand_in_called("Document::GetAllocator"); }
  Document& Parse(const char*) { json_stand_in_called("Document::Parse"); }
  template <class H>
  bool Accept(H&) const { json_stand_in_called("Document::Accept"); }
};

class StringBuffer {
 public:
  const char* GetString() const { json_stand_in_called("StringBuffer::GetString"); }
};

template <class OutputStream, class... Rest>
class Writer {
 public:
  explicit Writer(OutputStream&) {}
};

}  // namespace rapidjson
