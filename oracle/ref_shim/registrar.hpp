/* TEST INFRASTRUCTURE ONLY: the reference's factory-registration macros expand to nothing here. */
#pragma once
#define REGISTER_WITHOUT_ARGUMENTS(...)
#define REGISTER(...)
#define REGISTER_DEFAULT(...)
