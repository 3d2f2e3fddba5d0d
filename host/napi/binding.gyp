{
  "targets": [
    {
      "target_name": "closim_cuda",
      "sources": ["addon.cc"],
      "include_dirs": ["../../include"],
      "cflags_cc": ["-std=c++17", "-O2"],
      "libraries": ["-L<(module_root_dir)/../../closim_b200", "-lclosim_cuda",
                    "-Wl,-rpath,<(module_root_dir)/../../closim_b200"]
    }
  ]
}
