// Minimal stand-in for absl::Status where no absl installation exists (the
// backend adapter and the reference's CPU operators built in this repository;
// inside the reference's own tree its absl is used instead). It provides only
// what those use: status codes, code-plus-message construction,
// ok()/code()/message() and the *Error helper constructors.
#pragma once

#include <ostream>
#include <string>
#include <string_view>
#include <utility>

namespace absl {

using string_view = std::string_view;

enum class StatusCode : int {
  kOk = 0,
  kCancelled = 1,
  kUnknown = 2,
  kInvalidArgument = 3,
  kDeadlineExceeded = 4,
  kNotFound = 5,
  kAlreadyExists = 6,
  kPermissionDenied = 7,
  kResourceExhausted = 8,
  kFailedPrecondition = 9,
  kAborted = 10,
  kOutOfRange = 11,
  kUnimplemented = 12,
  kInternal = 13,
  kUnavailable = 14,
  kDataLoss = 15,
  kUnauthenticated = 16,
};

class Status {
 public:
  Status() = default;
  Status(StatusCode code, std::string_view message) : code_(code), message_(message) {}
  bool ok() const { return code_ == StatusCode::kOk; }
  StatusCode code() const { return code_; }
  int raw_code() const { return static_cast<int>(code_); }
  std::string_view message() const { return message_; }
  std::string ToString() const { return std::to_string(raw_code()) + ":" + message_; }
  friend bool operator==(const Status& a, const Status& b) { return a.code_ == b.code_ && a.message_ == b.message_; }
  friend bool operator!=(const Status& a, const Status& b) { return !(a == b); }
  void IgnoreError() const {}

 private:
  StatusCode code_ = StatusCode::kOk;
  std::string message_;
};

inline std::ostream& operator<<(std::ostream& os, const Status& s) { return os << s.ToString(); }

inline Status OkStatus() { return Status(); }
#define FL_SHIM_ERROR(Name, Code) \
  inline Status Name(std::string_view message) { return Status(StatusCode::Code, message); }
FL_SHIM_ERROR(InvalidArgumentError, kInvalidArgument)
FL_SHIM_ERROR(OutOfRangeError, kOutOfRange)
FL_SHIM_ERROR(ResourceExhaustedError, kResourceExhausted)
FL_SHIM_ERROR(FailedPreconditionError, kFailedPrecondition)
FL_SHIM_ERROR(InternalError, kInternal)
FL_SHIM_ERROR(AbortedError, kAborted)
FL_SHIM_ERROR(UnimplementedError, kUnimplemented)
FL_SHIM_ERROR(NotFoundError, kNotFound)
FL_SHIM_ERROR(UnavailableError, kUnavailable)
FL_SHIM_ERROR(DataLossError, kDataLoss)
FL_SHIM_ERROR(CancelledError, kCancelled)
FL_SHIM_ERROR(UnknownError, kUnknown)
FL_SHIM_ERROR(AlreadyExistsError, kAlreadyExists)
FL_SHIM_ERROR(DeadlineExceededError, kDeadlineExceeded)
#undef FL_SHIM_ERROR

inline bool IsInvalidArgument(const Status& s) { return s.code() == StatusCode::kInvalidArgument; }
inline bool IsOutOfRange(const Status& s) { return s.code() == StatusCode::kOutOfRange; }
inline bool IsFailedPrecondition(const Status& s) { return s.code() == StatusCode::kFailedPrecondition; }
inline bool IsResourceExhausted(const Status& s) { return s.code() == StatusCode::kResourceExhausted; }
inline bool IsInternal(const Status& s) { return s.code() == StatusCode::kInternal; }
inline bool IsAborted(const Status& s) { return s.code() == StatusCode::kAborted; }

}  // namespace absl
