{
  "targets": [
    {
      "target_name": "hush_node",
      "sources": ["hush_node.c"],
      "include_dirs": ["../include"],
      "libraries": ["-L<(module_root_dir)/../hush_b200", "-lhush_b200",
                    "-Wl,-rpath,<(module_root_dir)/../hush_b200"],
      "cflags": ["-std=c11", "-Wall", "-Wextra"]
    }
  ]
}
