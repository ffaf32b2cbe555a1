// Test-harness stand-in: user_options.h only names these two types in
// declarations of the command-line parser, which the harness does not build.
#pragma once
namespace boost {
namespace program_options {
class options_description {};
class positional_options_description {};
}  // namespace program_options
}  // namespace boost
