// Headless stand-in for manager/header/file_manager.h (nothing on the solve path uses it).
#pragma once
